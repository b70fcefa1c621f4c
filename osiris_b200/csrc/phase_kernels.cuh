// Phase appearance after an accepted time step (FP64): the saturation
// pressure of a one-phase cell and the phase-state update built on it.
//
// PhaseCtrl / fPhaseCtrl (compsim/Do_Cycle.cpp:1558-1721) visit every cell of
// a continuum: an oil-only cell whose oil pressure is at or below 0.95 of its
// bubble pressure, or a gas-only cell whose gas pressure is at or below 0.95
// of its dew pressure, becomes two-phase with a saturation of 1e-3 for the
// new phase and the incipient composition of the saturation-pressure
// calculation; otherwise a vanished oil (gas) saturation makes the cell
// gas-only (oil-only).  Saturations are then renormalised.  The saturation
// pressure (Bubl_Succ / Dew_Succ and the fracture's fBubl_Succ / fDew_Succ,
// compsim/Minor_NR.cpp:491-2015) is a successive substitution on the
// K-values and the pressure, and, when that fails, a Newton iteration on the
// N fugacity equalities and the sum of the incipient composition with a
// dense (N+1)^2 solve.  One thread per cell; the work is independent per
// cell.
#pragma once
#include "osiris_b200.h"
#include "eos_device.cuh"
#include "grid_kernels.cuh"

namespace osr {

constexpr double kEnvBoundary = 0.95;   // PAHSE_ENV_BOUNDARY, compsim/Functions.h:11
constexpr double kEpsSatPC = 1e-3;      // EPS_SAT, compsim/Functions.h:226
constexpr double kEpsSatFrac = 0;       // EPS_SAT_FRAC, compsim/Functions.h:12
constexpr double kPZero = 1000000;      // PZERO, compsim/Functions.h:247
constexpr double kSXmTol = 1e-15;       // SXMTOL, compsim/Functions.h:251
constexpr double kXmTol = 1e-8;         // XMTOL, compsim/Functions.h:224
constexpr double kTrivK = 1e-6;         // TRIV_K, compsim/Functions.h:269
constexpr int kMaxMnrIter = 20;         // MAX_MNR_ITER, compsim/Functions.h:270
constexpr double kRgas = 8.3144621;     // RGAS
constexpr double kPressTol = 1000;      // PRESSTOL, compsim/Functions.h:249
constexpr int kMaxNrIter = 100;         // cap of the Newton saturation pressure (the reference has none)

// Mixing sums of one phase: Ca = sum_ij w_i w_j sqrt(a_i a_j)(1 - k_ij),
// Cb = sum_i w_i b_i.
template <int N>
__device__ inline void mix_sums(const GridFluid<N> &G, const double *w, double &Ca, double &Cb) {
    Ca = 0;
    Cb = 0;
    for (int i = 0; i < N; i++) {
        Cb += w[i] * G.f.b[i];
        for (int j = 0; j < N; j++) Ca += w[i] * w[j] * (G.sa[i] * G.sa[j] * G.f.bic[i * N + j]);
    }
}

// sum_j w_j sqrt(a_i a_j)(1 - k_ij)
template <int N>
__device__ inline double mix_row(const GridFluid<N> &G, const double *w, int i) {
    double t = 0;
    for (int j = 0; j < N; j++) t += w[j] * (G.sa[i] * G.sa[j] * G.f.bic[i * N + j]);
    return t;
}

// One phase at pressure P: A, B, U, W, Z and the scale factors.
struct PhaseEos {
    double Ca, Cb, A, B, U, W, Z;
};

template <int N>
__device__ inline PhaseEos phase_eos(const GridFluid<N> &G, const double *w, double P, bool gas) {
    PhaseEos e;
    mix_sums<N>(G, w, e.Ca, e.Cb);
    const double T = G.T;
    e.A = e.Ca * (P / (kRgas * kRgas * T * T));
    e.B = e.Cb * (P / (kRgas * T));
    const bool srk = G.f.srk;
    e.U = srk ? e.B : 2 * e.B;
    e.W = srk ? 0.0 : e.B;
    e.Z = solve_z(-(1 + e.B - e.U), e.A - e.B * e.U - e.U - e.W * e.W, -(e.A * e.B - e.B * e.W * e.W - e.W * e.W), gas);
    return e;
}

// Fugacity coefficient of component i in a phase (compsim/Init_Calcs.cpp:633-711).
template <int N>
__device__ inline double phase_phi(const GridFluid<N> &G, const PhaseEos &e, double ti, int i, double d1, double d2,
                                   double *EE, double *DD, double *FF) {
    const double t1 = G.f.b[i] / e.Cb;
    *EE = 2 * ti / e.Ca - t1;
    *DD = e.A / (e.B * (d1 - d2));
    *FF = log((e.Z + d2 * e.B) / (e.Z + d1 * e.B));
    return exp(t1 * (e.Z - 1) - log(e.Z - e.B) + *DD * *EE * *FF);
}

// dZ for changes dA, dB of A and B (U, W follow the EOS).
__device__ inline double dz_of(const PhaseEos &e, bool srk, double dA, double dB) {
    const double dU = srk ? dB : 2 * dB, dW = srk ? 0.0 : dB;
    const double Z = e.Z, B = e.B, U = e.U, W = e.W, A = e.A;
    return -(dA * (Z - B) + dB * (-Z * Z - U * Z - A + W * W) + dU * (Z * Z - B * Z - Z) + dW * (-2 * W * Z + 2 * B * W + 2 * W)) /
           (3 * Z * Z - 2 * Z * (1 + B - U) + A - B * U - U - W * W);
}

// Dense solve with partial pivoting, column by column (the dgesv the
// reference's MKLS calls, compsim/MKL_Solver.Cpp:66-90): a[i*n+k] is row i,
// column k; the solution replaces b.  A zero pivot leaves b as eliminated so
// far, as the reference's solve does.
__device__ inline void dense_solve(double *a, double *b, int n) {
    bool singular = false;
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++) {
            const double v = fabs(a[i * n + k]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (a[p * n + k] == 0.0) {
            singular = true;
            continue;
        }
        if (p != k) {
            for (int j = 0; j < n; j++) {
                const double t = a[k * n + j];
                a[k * n + j] = a[p * n + j];
                a[p * n + j] = t;
            }
            const double t = b[k];
            b[k] = b[p];
            b[p] = t;
        }
        const double piv = a[k * n + k];
        for (int i = k + 1; i < n; i++) {
            const double l = a[i * n + k] / piv;
            a[i * n + k] = l;
            for (int j = k + 1; j < n; j++) a[i * n + j] -= l * a[k * n + j];
            b[i] -= l * b[k];
        }
    }
    if (singular) return;
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int k = i + 1; k < n; k++) s -= a[i * n + k] * b[k];
        b[i] = s / a[i * n + i];
    }
}

// The Newton system of a saturation pressure in the unknowns (Xm, P): rows
// 0..N-1 the fugacity equalities wl_i phiL_i = wg_i phiG_i, row N the sum of
// the incipient composition; r receives minus the residual and J (row-major,
// (N+1)^2) its derivatives.  The bubble point's incipient phase is the gas
// (wl = own), the dew point's the liquid (wg = own).  The rows are those of
// Bubl_NR / Dew_NR (compsim/Minor_NR.cpp:76-252, :290-470) and of the Newton
// fallback inside Bubl_Succ / Dew_Succ.
template <int N>
__device__ inline void sat_newton_system(const GridFluid<N> &G, bool dew, const double *own, const double *Xm, double P,
                                         double *J, double *r) {
    constexpr int M = N + 1;
    const bool srk = G.f.srk;
    const double d1 = srk ? 1.0 : 1 + 1.4142135623730950488016887, d2 = srk ? 0.0 : 1 - 1.4142135623730950488016887;
    const double T = G.T;
    double SXm = 0;
    for (int i = 0; i < N; i++) {
        SXm += Xm[i];
        J[N * M + i] = 1;
    }
    r[N] = -SXm + 1;
    J[N * M + N] = 0;
    const double *wl = dew ? Xm : own, *wg = dew ? own : Xm;
    const PhaseEos el = phase_eos<N>(G, wl, P, false), eg = phase_eos<N>(G, wg, P, true);
    const PhaseEos &ei = dew ? el : eg;   // the incipient phase
    const double RRT = kRgas * kRgas * T * T, RT = kRgas * T;
    const double dZdpl = dz_of(el, srk, el.Ca / RRT, el.Cb / RT);
    const double dZdpg = dz_of(eg, srk, eg.Ca / RRT, eg.Cb / RT);
    for (int i = 0; i < N; i++) {
        const double tl = mix_row<N>(G, wl, i), tg = mix_row<N>(G, wg, i);
        double EEl, DDl, FFl, EEg, DDg, FFg;
        const double phiL = phase_phi<N>(G, el, tl, i, d1, d2, &EEl, &DDl, &FFl);
        const double phiG = phase_phi<N>(G, eg, tg, i, d1, d2, &EEg, &DDg, &FFg);
        r[i] = -wl[i] * phiL + wg[i] * phiG;
        // pressure derivatives of both coefficients
        const double bi = G.f.b[i];
        const double dAdpl = el.Ca / RRT, dBdpl = el.Cb / RT, dAdpg = eg.Ca / RRT, dBdpg = eg.Cb / RT;
        const double dAAdpl = bi * dZdpl / el.Cb, dAAdpg = bi * dZdpg / eg.Cb;
        const double dBBdpl = (dBdpl - dZdpl) / (el.Z - el.B), dBBdpg = (dBdpg - dZdpg) / (eg.Z - eg.B);
        const double dDDdpl = (el.B * dAdpl - el.A * dBdpl) / (el.B * el.B * (d1 - d2));
        const double dDDdpg = (eg.B * dAdpg - eg.A * dBdpg) / (eg.B * eg.B * (d1 - d2));
        const double dFFdpl = (dZdpl + d2 * dBdpl) / (el.Z + d2 * el.B) - (dZdpl + d1 * dBdpl) / (el.Z + d1 * el.B);
        const double dFFdpg = (dZdpg + d2 * dBdpg) / (eg.Z + d2 * eg.B) - (dZdpg + d1 * dBdpg) / (eg.Z + d1 * eg.B);
        const double dPhidpl = phiL * (dAAdpl + dBBdpl + EEl * (dDDdpl * FFl + DDl * dFFdpl));
        const double dPhidpg = phiG * (dAAdpg + dBBdpg + EEg * (dDDdpg * FFg + DDg * dFFdpg));
        J[i * M + N] = wl[i] * dPhidpl - wg[i] * dPhidpg;
        // derivatives with respect to the incipient composition
        const double ti = dew ? tl : tg, phi = dew ? phiL : phiG;
        const double EE = dew ? EEl : EEg, DD = dew ? DDl : DDg, FF = dew ? FFl : FFg;
        for (int kk = 0; kk < N; kk++) {
            double dAdx = 0;
            for (int n = 0; n < N; n++) dAdx += Xm[n] * (G.sa[n] * G.sa[kk] * G.f.bic[n * N + kk]);
            dAdx *= 2 * P / RRT;
            const double dBdx = G.f.b[kk] * P / RT;
            const double dZdx = dz_of(ei, srk, dAdx, dBdx);
            const double dAAdx = -G.f.b[kk] * bi * (ei.Z - 1) / (ei.Cb * ei.Cb) + bi * dZdx / ei.Cb;
            const double dBBdx = (dBdx - dZdx) / (ei.Z - ei.B);
            const double dDDdx = (dAdx * ei.B - dBdx * ei.A) / (ei.B * ei.B * (d1 - d2));
            const double dFFdx = (dZdx + d2 * dBdx) / (ei.Z + d2 * ei.B) - (dZdx + d1 * dBdx) / (ei.Z + d1 * ei.B);
            const double dEEdx = 2 * (G.f.bic[i * N + kk] * (G.sa[i] * G.sa[kk]) / ei.Ca - dAdx * RRT * ti / (P * ei.Ca * ei.Ca)) +
                                 bi * G.f.b[kk] / (ei.Cb * ei.Cb);
            const double dPhidx = phi * (dAAdx + dBBdx + dDDdx * EE * FF + DD * dEEdx * FF + DD * EE * dFFdx);
            if (dew) J[i * M + kk] = i == kk ? phi + Xm[i] * dPhidx : Xm[i] * dPhidx;
            else J[i * M + kk] = i == kk ? -phi - Xm[i] * dPhidx : -Xm[i] * dPhidx;
        }
    }
}

// Saturation pressure of a one-phase cell: bubble (dew = false; x the oil
// composition, P0 the oil pressure) or dew (dew = true; y the gas
// composition, P0 the gas pressure).  seed: the cell's vapour composition,
// from which the reference's substitution starts in both cases.  Returns the
// pressure, or -1 where the reference's function returns -1 (iteration cap,
// trivial solution); Xm receives the incipient phase's composition.
template <int N>
__device__ double sat_pressure(const GridFluid<N> &G, bool dew, const double *own, const double *seed, double P0,
                               double *Xm) {
    const bool srk = G.f.srk;
    const double d1 = srk ? 1.0 : 1 + 1.4142135623730950488016887, d2 = srk ? 0.0 : 1 - 1.4142135623730950488016887;
    const double T = G.T;
    // successive substitution on K and P
    double P = P0;
    double K[N];
    for (int i = 0; i < N; i++) K[i] = (G.f.pc[i] / P) * exp(G.f.wil[i] * (1 - G.f.tc[i] / T));
    bool fail = false;
    int it = 0, k = 0;
    double SXm = 0, sumK = 0;
    do {
        double xs = 0;
        for (int i = 0; i < N; i++) {
            double v = seed[i] / K[i];
            if (v < 0) v = 0;
            else if (v > 1) v = 1;
            Xm[i] = v;
            xs += v;
        }
        if (P < 0) P = kPZero;
        for (int i = 0; i < N; i++) Xm[i] /= xs;
        const double *wl = dew ? Xm : own, *wg = dew ? own : Xm;
        const PhaseEos el = phase_eos<N>(G, wl, P, false), eg = phase_eos<N>(G, wg, P, true);
        SXm = 0;
        k = 0;
        sumK = 0;
        for (int i = 0; i < N; i++) {
            double EE, DD, FF;
            const double phiL = phase_phi<N>(G, el, mix_row<N>(G, wl, i), i, d1, d2, &EE, &DD, &FF);
            const double phiG = phase_phi<N>(G, eg, mix_row<N>(G, wg, i), i, d1, d2, &EE, &DD, &FF);
            const double fL = wl[i] * phiL, fG = wg[i] * phiG;
            if (own[i] != 0) {
                K[i] *= fL / fG;
                SXm += dew ? own[i] / K[i] : K[i] * own[i];
                sumK += fabs(1 - K[i]);
                k++;
            }
        }
        P *= SXm;
        it++;
        if (it > kMaxMnrIter) {
            fail = true;
            break;
        }
    } while ((fabs(SXm - 1) / k) > kSXmTol);
    if ((sumK / k) < kTrivK) fail = true;
    if (!fail && (P - P) == 0) return P;

    // Newton on [fugacity equalities; sum of Xm = 1] in (Xm, P)
    constexpr int M = N + 1;
    double J[M * M], r[M], x[M];
    P = P0;
    for (int i = 0; i < N; i++) {
        const double NRKi = (G.f.pc[i] / P) * exp(G.f.wil[i] * (1 - G.f.tc[i] / T));
        Xm[i] = dew ? own[i] / NRKi : NRKi * own[i];
    }
    it = 0;
    double XmTol;
    do {
        sat_newton_system<N>(G, dew, own, Xm, P, J, r);
        dense_solve(J, r, M);
        for (int i = 0; i < M; i++) x[i] = r[i];
        XmTol = 0;
        double xs = 0;
        for (int i = 0; i < M; i++) {
            double &v = i < N ? Xm[i] : P;
            v += x[i];
            if (i < N) {
                if (v < 0) v = 0;
                else if (v > 1) v = 1;
                xs += v;
            } else if (v < 0) {
                v = kPZero;
            }
            XmTol += v != 0 ? fabs(x[i] / v) : fabs(x[i]);
        }
        XmTol /= M;
        for (int i = 0; i < N; i++) Xm[i] /= xs;
        it++;
        if (it > kMaxMnrIter) return -1;
    } while (XmTol > kXmTol);
    sumK = 0;
    k = 0;
    for (int i = 0; i < N; i++) {
        if (own[i] != 0) {
            sumK += dew ? fabs(1 - own[i] / Xm[i]) : fabs(1 - Xm[i] / own[i]);
            k++;
        }
    }
    if ((sumK / k) < kTrivK) return -1;
    return P;
}

// The saturation pressure of every one-phase cell of one continuum (0 for
// two-phase cells) and its incipient composition.
template <int N>
__global__ void __launch_bounds__(128) sat_pressure_kernel(const __grid_constant__ GridArgs<N> a, int med,
                                                           double *psat, double *xm) {
    const MediumFields &F = a.m[med];
    const long n = a.s.cells;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int lab = F.label[c];
        double x[N], y[N], X[N];
        for (int i = 0; i < N; i++) {
            x[i] = F.x[(long)i * n + c];
            y[i] = F.y[(long)i * n + c];
            X[i] = 0;
        }
        double p = 0;
        if (lab == 1) p = sat_pressure<N>(a.g, false, x, y, F.P[n + c], X);
        else if (lab == -1) p = sat_pressure<N>(a.g, true, y, y, F.P[2 * n + c], X);
        psat[c] = p;
        if (xm)
            for (int i = 0; i < N; i++) xm[(long)i * n + c] = X[i];
    }
}

// PhaseCtrl (matrix, med = 0) / fPhaseCtrl (fracture, med = 1) on every cell.
template <int N>
__global__ void __launch_bounds__(128) phase_ctrl_kernel(const __grid_constant__ GridArgs<N> a) {
    const int med = blockIdx.y;
    const MediumFields &F = a.m[med];
    const long n = a.s.cells;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        int lab = F.label[c];
        double S0 = F.sat[c], S1 = F.sat[n + c], S2 = F.sat[2 * n + c];
        double x[N], y[N], X[N];
        for (int i = 0; i < N; i++) {
            x[i] = F.x[(long)i * n + c];
            y[i] = F.y[(long)i * n + c];
        }
        bool appeared = false;
        if (lab == -1 && F.P[2 * n + c] <= kEnvBoundary * sat_pressure<N>(a.g, true, y, y, F.P[2 * n + c], X)) {
            S1 = kEpsSatPC;
            S2 -= kEpsSatPC;
            lab = 0;
            for (int i = 0; i < N; i++) F.x[(long)i * n + c] = X[i];
            appeared = true;
        } else if (lab == 1 && F.P[n + c] <= kEnvBoundary * sat_pressure<N>(a.g, false, x, y, F.P[n + c], X)) {
            S2 = kEpsSatPC;
            S1 -= kEpsSatPC;
            lab = 0;
            for (int i = 0; i < N; i++) F.y[(long)i * n + c] = X[i];
            appeared = true;
        }
        if (!appeared) {
            if (S1 <= kEpsSatPC * kEpsSatFrac) {
                S1 = 0;
                S2 = 1 - S0;
                lab = -1;
            }
            if (S2 <= kEpsSatPC * kEpsSatFrac) {
                S2 = 0;
                S1 = 1 - S0;
                lab = 1;
            }
        }
        const double norm = 1.0 / (S0 + S1 + S2);
        F.sat[c] = S0 * norm;
        F.sat[n + c] = S1 * norm;
        F.sat[2 * n + c] = S2 * norm;
        F.label[c] = (signed char)lab;
    }
}

// ---------------------------------------------------------------------------
// Newton saturation pressure, lower dew point and the SS-flash stability test
// (compsim/Minor_NR.cpp:33-489, 2017-2308).  The reference keeps these with
// their call sites commented out (compsim/Do_Cycle.cpp:1576-1605, 1653-1682,
// compsim/Do_Time_Step.cpp:404); here they are opt-in entry points.
// ---------------------------------------------------------------------------

// Bubl_NR (dew = false; own = the oil composition, P0 = the oil pressure) and
// Dew_NR (dew = true; own = the gas composition, P0 = the gas pressure),
// compsim/Minor_NR.cpp:33-266 / 268-489: Newton on the saturation-pressure
// system from the Wilson K-values at P0.  Before each step the incipient
// composition is clamped to [0, 1] (not renormalised) and a negative pressure
// is reset to 1e6 Pa; the iteration ends once the mean of |step / value| over
// the N + 1 unknowns is at most 1e-8 or the pressure step at most 1000 Pa.
// The reference iterates without a cap; here a cell stops after kMaxNrIter
// steps with OSR_CELL_MAXIT.  Xm and *Pout receive the last iterate.
template <int N>
__device__ int sat_pressure_nr(const GridFluid<N> &G, bool dew, const double *own, double P0, double *Xm, double *Pout,
                               int *iters) {
    constexpr int M = N + 1;
    double J[M * M], r[M];
    double P = P0;
    for (int i = 0; i < N; i++) {
        const double NRKi = (G.f.pc[i] / P) * exp(G.f.wil[i] * (1 - G.f.tc[i] / G.T));
        Xm[i] = dew ? own[i] / NRKi : NRKi * own[i];
    }
    int it = 0, st = OSR_CELL_OK;
    for (;;) {
        for (int i = 0; i < N; i++) {
            if (Xm[i] < 0) Xm[i] = 0;
            else if (Xm[i] > 1) Xm[i] = 1;
        }
        if (P < 0) P = kPZero;
        sat_newton_system<N>(G, dew, own, Xm, P, J, r);
        dense_solve(J, r, M);
        double XmTol = 0;
        for (int i = 0; i < M; i++) {
            double &v = i < N ? Xm[i] : P;
            v += r[i];
            XmTol += fabs(r[i] / v);
        }
        XmTol /= M;
        it++;
        if (!((XmTol > kXmTol) && (fabs(r[N]) > kPressTol))) break;
        if (it >= kMaxNrIter) {
            st = OSR_CELL_MAXIT;
            break;
        }
    }
    *Pout = P;
    *iters = it;
    if (st == OSR_CELL_OK && !(P - P == 0)) st = OSR_CELL_NAN;
    return st;
}

// LowerDew_Succ (compsim/Minor_NR.cpp:2017-2136): the lower dew point of a
// gas-only cell by successive substitution from the Wilson K-values at the
// gas pressure.  Each step sets the liquid composition to y / K clamped to
// [0, 1] (not renormalised), updates K by the fugacity ratio of the
// components present and divides the pressure by sum(y / K); at most 21
// steps, ending once |sum(y / K) - 1| / n <= 1e-15.  A trivial solution
// (mean |1 - K| < 1e-6) returns 1e100.  Xm receives the liquid composition of
// the last step.
template <int N>
__device__ double lower_dew(const GridFluid<N> &G, const double *own, double P0, double *Xm, int *iters) {
    const bool srk = G.f.srk;
    const double d1 = srk ? 1.0 : 1 + 1.4142135623730950488016887, d2 = srk ? 0.0 : 1 - 1.4142135623730950488016887;
    double P = P0;
    double K[N];
    for (int i = 0; i < N; i++) K[i] = (G.f.pc[i] / P) * exp(G.f.wil[i] * (1 - G.f.tc[i] / G.T));
    int it = 0, k = 0;
    double SXm = 0, sumK = 0;
    do {
        for (int i = 0; i < N; i++) {
            double v = own[i] / K[i];
            if (v < 0) v = 0;
            else if (v > 1) v = 1;
            Xm[i] = v;
        }
        if (P < 0) P = 1;
        const PhaseEos el = phase_eos<N>(G, Xm, P, false), eg = phase_eos<N>(G, own, P, true);
        SXm = 0;
        k = 0;
        sumK = 0;
        for (int i = 0; i < N; i++) {
            double EE, DD, FF;
            const double phiL = phase_phi<N>(G, el, mix_row<N>(G, Xm, i), i, d1, d2, &EE, &DD, &FF);
            const double phiG = phase_phi<N>(G, eg, mix_row<N>(G, own, i), i, d1, d2, &EE, &DD, &FF);
            const double fL = Xm[i] * phiL, fG = own[i] * phiG;
            if (own[i] != 0) {
                K[i] *= fL / fG;
                SXm += own[i] / K[i];
                sumK += fabs(1 - K[i]);
                k++;
            }
        }
        P /= SXm;
        it++;
        if (it > kMaxMnrIter) break;
    } while ((fabs(SXm - 1) / k) > kSXmTol);
    *iters = it;
    if ((sumK / k) < kTrivK) P = 1e100;
    return P;
}

// critTest (compsim/Minor_NR.cpp:2138-2308): the stability test of a
// one-phase cell.  The cell's own composition (oil for an oil-only cell, gas
// for a gas-only cell) is flashed at the oil pressure by successive
// substitution from Wilson K-values: each outer step runs a Rachford-Rice
// Newton from L = 0.5 (at most 100 steps, step^2 <= 1e-8; a K below zero
// marks a component that stays in the gas), clamps L to [0, 1], forms
// x = z / (L + K (1 - L)), y = K x and updates K by the fugacity ratio (a
// zero or NaN gas fugacity sets K = -1, a NaN liquid fugacity K = -1, a NaN
// gas fugacity K = 1).  It ends once L moves by at most 1e-14, or after 21
// steps.  An oil-only cell whose L reaches 0 becomes gas-only (gas
// composition = its oil composition, gas saturation = its oil saturation);
// a gas-only cell whose L reaches 1 becomes oil-only.  Returns whether the
// label changed.
template <int N>
__device__ bool crit_test(const GridFluid<N> &G, int lab, const double *z, double Po, double *Lout, int *iters) {
    const bool srk = G.f.srk;
    const double d1 = srk ? 1.0 : 1 + 1.4142135623730950488016887, d2 = srk ? 0.0 : 1 - 1.4142135623730950488016887;
    double K[N], xs[N], ys[N];
    for (int i = 0; i < N; i++) K[i] = (G.f.pc[i] / Po) * exp(G.f.wil[i] * (1 - G.f.tc[i] / G.T));
    int nIter = 0;
    double L = 0.5, Lb = 10, ESum;
    do {
        L = 0.5;
        int j = 0;
        double step;
        do {
            double F = 0, dF = 0;
            for (int i = 0; i < N; i++) {
                const double t = K[i] >= 0 ? (1 - K[i]) / (L + (1 - L) * K[i]) : 1 / (L - 1);
                F += z[i] * t;
                dF -= z[i] * t * t;
            }
            step = F / dF;
            L -= step;
            j++;
        } while ((step * step > kRRTol) && (j < kRRMaxIt));
        if (L > 1) L = 1;
        else if (L < 0) L = 0;
        ESum = fabs(Lb - L);
        Lb = L;
        for (int i = 0; i < N; i++) {
            if (K[i] >= 0) {
                xs[i] = z[i] / (L + K[i] * (1 - L));
                ys[i] = K[i] * xs[i];
            } else {
                xs[i] = 0;
                ys[i] = z[i] / (1 - L);
            }
        }
        const PhaseEos el = phase_eos<N>(G, xs, Po, false), eg = phase_eos<N>(G, ys, Po, true);
        for (int i = 0; i < N; i++) {
            double EE, DD, FF;
            const double phiL = phase_phi<N>(G, el, mix_row<N>(G, xs, i), i, d1, d2, &EE, &DD, &FF);
            const double phiG = phase_phi<N>(G, eg, mix_row<N>(G, ys, i), i, d1, d2, &EE, &DD, &FF);
            const double fL = xs[i] * phiL, fG = ys[i] * phiG;
            if (z[i] != 0) {
                if (fG != 0) K[i] *= fL / fG;
                else K[i] = -1;
                if (fL != fL) K[i] = -1;
                if (fG != fG) K[i] = 1;
            }
        }
        nIter++;
        if (nIter > kMaxMnrIter) break;
    } while (ESum > kSSTol);
    *Lout = L;
    *iters = nIter;
    return (fabs(L) < kLZero && lab == 1) || (fabs(1 - L) < kLZero && lab == -1);
}

// Bubl_NR (kind 0, oil-only cells), Dew_NR (kind 1, gas-only cells) or
// LowerDew_Succ (kind 2, gas-only cells) on every cell of one continuum.
// Other cells get pressure 0, composition 0 and status OK.
template <int N>
__global__ void __launch_bounds__(128) sat_pressure_nr_kernel(const __grid_constant__ GridArgs<N> a, int med, int kind,
                                                              double *psat, double *xm, int *status, int *iters) {
    const MediumFields &F = a.m[med];
    const long n = a.s.cells;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int lab = F.label[c];
        double own[N], X[N];
        for (int i = 0; i < N; i++) X[i] = 0;
        double p = 0;
        int st = OSR_CELL_OK, it = 0;
        if (kind == 0 && lab == 1) {
            for (int i = 0; i < N; i++) own[i] = F.x[(long)i * n + c];
            st = sat_pressure_nr<N>(a.g, false, own, F.P[n + c], X, &p, &it);
        } else if (kind != 0 && lab == -1) {
            for (int i = 0; i < N; i++) own[i] = F.y[(long)i * n + c];
            if (kind == 1) {
                st = sat_pressure_nr<N>(a.g, true, own, F.P[2 * n + c], X, &p, &it);
            } else {
                p = lower_dew<N>(a.g, own, F.P[2 * n + c], X, &it);
                if (!(p - p == 0)) st = OSR_CELL_NAN;
            }
        }
        psat[c] = p;
        if (xm)
            for (int i = 0; i < N; i++) xm[(long)i * n + c] = X[i];
        if (status) status[c] = st;
        if (iters) iters[c] = it;
    }
}

// critTest on every one-phase cell of one continuum; relabels the cells it
// finds in the other phase and counts them in *changed.
template <int N>
__global__ void __launch_bounds__(128) crit_test_kernel(const __grid_constant__ GridArgs<N> a, int med, double *lout,
                                                        int *changed) {
    const MediumFields &F = a.m[med];
    const long n = a.s.cells;
    int mine = 0;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int lab = F.label[c];
        double L = -1;
        if (lab == 1 || lab == -1) {
            const double *src = lab == 1 ? F.x : F.y;
            double z[N];
            for (int i = 0; i < N; i++) z[i] = src[(long)i * n + c];
            int it;
            if (crit_test<N>(a.g, lab, z, F.P[n + c], &L, &it)) {
                if (lab == 1) {
                    for (int i = 0; i < N; i++) F.y[(long)i * n + c] = z[i];
                    F.sat[2 * n + c] = F.sat[n + c];
                    F.sat[n + c] = 0;
                    F.label[c] = -1;
                } else {
                    for (int i = 0; i < N; i++) F.x[(long)i * n + c] = z[i];
                    F.sat[n + c] = F.sat[2 * n + c];
                    F.sat[2 * n + c] = 0;
                    F.label[c] = 1;
                }
                mine++;
            }
        }
        if (lout) lout[c] = L;
    }
    if (changed) {
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        if ((threadIdx.x & 31) == 0 && mine) atomicAdd(changed, mine);
    }
}

}  // namespace osr
