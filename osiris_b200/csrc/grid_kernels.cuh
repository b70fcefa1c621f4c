// Per-cell property sweeps of a dual-porosity grid (FP64, sm_100a).
//
// One kernel evaluates, for every cell of both continua, the chain the
// reference runs cell by cell in UpdateDependencies
// (compsim/PetscAUX.cpp:530-548): interfacial tension from the previous
// densities, relative permeabilities and capillary pressures, phase
// pressures, densities with their composition/pressure derivatives and LBC
// viscosities, accumulation at the linearisation point, Sigmund diffusion
// coefficients and phase gravity.  A second kernel evaluates the
// upstream-weighted transmissibilities of each cell's +x, +y, +z faces
// (Calc_Transes / fCalc_Transes).  Fields are structure-of-arrays with the
// cell index (i + nx*(j + ny*k)) fastest.
#pragma once
#include "eos_device.cuh"

namespace osr {

constexpr double kGAcc = 9.80665;        // G_ACC, compsim/Functions.h:198
constexpr double kGAccG = 9.80665e-3;    // G_ACCG, compsim/Functions.h:199
constexpr double kWatMRo = 55.5084;      // WAT_M_RO, compsim/Functions.h:206
constexpr double kIftBase = 50;          // IFTBASECASE, compsim/Functions.h:279
constexpr double kIftPower = 7;          // IFTPOWER, compsim/Functions.h:280
constexpr double kMiscibleIft = 1;       // MISCIBLEIFT, compsim/Functions.h:281
constexpr double kEpsSat = 1e-3;         // EPS_SAT, compsim/Functions.h:226

// Per-component constants of a grid model at the reservoir temperature.
template <int N>
struct GridFluid {
    FluidTable<N> f;
    double sa[N];        // sqrt(a_i(T_res))
    double mw[N];        // molecular weight
    double smw[N];       // sqrt(mw)
    double mui[N];       // dilute-gas viscosity (Tr_Mu, compsim/Init_Calcs.cpp:48-64)
    double vcm[N];       // critical volume after the reference's /1e6 (m3/mol)
    double pcr_atm[N];   // Pc / 101325
    double vc53[N];      // vcm^(5/3)
    double vc23[N];      // vcm^(2/3)
    double parachor[N];
    double pD[N * N];    // binary diffusion factor pDij (compsim/Mass_Tran.cpp:43-46)
    double pDlast[N];    // pDij of the last k != j (used when w_j == 1)
    double T;            // reservoir temperature [K]
};

// Scalars and small tables of the model.
struct GridScalars {
    int nx, ny, nz;
    long cells;
    double wat_ro, wat_mu, refp, cpor, dcpor;
    int const_dif;       // CDIF present
    double cdif;
    const double *swt, *sgt;  // [n][4] device
    int nswt, nsgt;
};

// Device fields of one continuum (medium).  Per-cell [cells]; multi-valued
// fields are [k][cells].
struct MediumFields {
    double *P;       // [3] water, oil, gas pressure
    double *sat;     // [3]
    double *x, *y, *z;  // [nc]
    signed char *label;
    double *rho, *pc, *mu, *gam;  // [2]
    double *kr;      // [3]
    double *dkr;     // [5]
    double *dE;      // [(nc+1)*2]  (component or pressure, phase)
    double *pre;     // [nc+1]
    double *diff;    // [nc*2]
    double *ift;     // [1]
    double *trans;   // [12*3]
    signed char *transS;  // [3*3]
    double *wtran, *dwtran;  // [3]
    double *por;     // [1]
    double *perm;    // [3]
    double *iftran;  // [3]
};

struct GridGeom {
    const double *di, *dj, *dk;  // [nx], [ny], [nz]
    const double *blockH;        // [cells]
};

template <int N>
struct GridArgs {
    GridFluid<N> g;
    GridScalars s;
    GridGeom geo;
    MediumFields m[2];   // 0 = matrix, 1 = fracture
};

// Piecewise-linear table lookup of the reference (first row with s < S_n).
struct TableHit {
    double kr, krx, pc, dkr, dkrx;
};

__device__ __forceinline__ TableHit table_lookup(const double *t, int n, double s) {
    // t[row*4 + col]: col 0 saturation, 1 kr, 2 kro, 3 Pc
    int r = 0;
    while (r < n && !(s < t[r * 4])) r++;
    TableHit h;
    if (r == 0) {
        h.kr = 0;  // RELPERM0
        h.pc = t[3];
        h.krx = t[2];
        h.dkr = 0;
        h.dkrx = 0;
    } else if (r == n) {
        h.kr = t[(n - 1) * 4 + 1];
        h.pc = t[(n - 1) * 4 + 3];
        h.krx = t[(n - 1) * 4 + 2];
        h.dkr = 0;
        h.dkrx = 0;
    } else {
        // slope * (s - s_r) + v_r with the product rounded before the add, as
        // the reference compiles it: at a table node the two terms cancel to
        // exactly 0 (a fused multiply-add would leave a 1e-19 residue there).
        const double *a = t + (r - 1) * 4, *b = t + r * 4;
        double ds = b[0] - a[0], dsb = s - b[0];
        h.dkr = (b[1] - a[1]) / ds;
        h.dkrx = (b[2] - a[2]) / ds;
        h.kr = __dadd_rn(__dmul_rn(h.dkr, dsb), b[1]);
        h.krx = __dadd_rn(__dmul_rn(h.dkrx, dsb), b[2]);
        h.pc = __dadd_rn(__dmul_rn((b[3] - a[3]) / ds, dsb), b[3]);
    }
    return h;
}

// Density, its composition/pressure derivatives and the LBC viscosity of one
// phase (Calc_Visco, compsim/Do_Cycle.cpp:460-614).  w: composition, P: the
// phase's pressure.  dE[k] = d rho / d w_k, dE[N] = d rho / d P.
template <int N>
__device__ __forceinline__ void phase_density_visc(const GridFluid<N> &g, const double *w, double P, bool gas,
                                                   double &rho, double &mu, double *dE) {
    const FluidTable<N> &f = g.f;
    const double T = g.T;
    double u[N], v[N];
#pragma unroll
    for (int i = 0; i < N; i++) u[i] = w[i] * g.sa[i];
    double Ca = 0, Cb = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < N; j++) s += f.bic[i * N + j] * u[j];
        v[i] = s;
        Ca += u[i] * s;
        Cb += w[i] * f.b[i];
    }
    const double rt = kR * T;
    double A = Ca * (P / (rt * rt)), B = Cb * (P / rt);
    double dAdp = Ca / (rt * rt), dBdp = Cb / rt;
    const bool srk = f.srk != 0;
    double U = srk ? B : 2 * B, W = srk ? 0.0 : B;
    double dUdp = srk ? dBdp : 2 * dBdp, dWdp = srk ? 0.0 : dBdp;
    double Z = solve_z(-(1 + B - U), A - B * U - U - W * W, -(A * B - B * W * W - W * W), gas);
    double cA = Z - B, cB = -Z * Z - U * Z - A + W * W, cU = Z * Z - B * Z - Z, cW = -2 * W * Z + 2 * B * W + 2 * W;
    double den = 3 * Z * Z - 2 * Z * (1 + B - U) + A - B * U - U - W * W;
    double dZdp = -(dAdp * cA + dBdp * cB + dUdp * cU + dWdp * cW) / den;
    dE[N] = (1 - P * dZdp / Z) / (rt * Z);
    const double twopa = 2 * P / (rt * rt), pb = P / rt;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double dA = g.sa[k] * v[k] * twopa;
        double dB = f.b[k] * pb;
        double dU = srk ? dB : 2 * dB, dW = srk ? 0.0 : dB;
        double dZ = -(dA * cA + dB * cB + dU * cU + dW * cW) / den;
        dE[k] = -(P * dZ / (rt * Z * Z));
    }
    rho = P / (Z * rt);
    double s1 = 0, s2 = 0, ro = 0, tcm = 0, pcm = 0, mwm = 0;
#pragma unroll
    for (int n = 0; n < N; n++) {
        double t = w[n] * g.smw[n];
        s1 += t * g.mui[n];
        s2 += t;
        ro += w[n] * g.vcm[n];
        tcm += w[n] * f.tc[n];
        pcm += w[n] * g.pcr_atm[n];
        mwm += w[n] * g.mw[n];
    }
    double Er = rho * ro;
    double eta = pow(tcm, 1.0 / 6) / (sqrt(mwm) * pow(pcm, 2.0 / 3));
    double r1 = 0.10230 + 0.023364 * Er + 0.058533 * Er * Er - 0.040758 * Er * Er * Er + 0.0093324 * Er * Er * Er * Er;
    mu = s1 / s2 + (r1 * r1 * r1 * r1 - 1e-4) / eta;
}

// Effective diffusion coefficients of one phase (CalcDiffusion,
// compsim/Mass_Tran.cpp:29-56).
template <int N>
__device__ __forceinline__ void phase_diffusion(const GridFluid<N> &g, const GridScalars &s, const double *w,
                                                double rho, double *D) {
    double s1 = 0, s2 = 0;
#pragma unroll
    for (int j = 0; j < N; j++) {
        s1 += w[j] * g.vc53[j];
        s2 += w[j] * g.vc23[j];
    }
    s1 = rho * s1 / s2;
    double roRD = (0.99589 + 0.096016 * s1 - 0.22035 * s1 * s1 + 0.032874 * s1 * s1 * s1) / rho;
#pragma unroll
    for (int j = 0; j < N; j++) {
        double sum = 0;
#pragma unroll
        for (int k = 0; k < N; k++)
            if (k != j) sum += w[k] / (g.pD[j * N + k] * roRD);
        double dt = (1 - w[j]) / (sum * 10000);
        double d;
        if (w[j] == 1) d = roRD * g.pDlast[j];
        else if ((dt < 0) || (sum == 0)) d = 0;
        else d = dt;  // DIFF_INTERNAL_COEFF = 1
        if (s.const_dif) d = s.cdif;
        D[j] = d;
    }
}

// The per-cell chain of UpdateDependencies for one medium.
template <int N>
__global__ void __launch_bounds__(128) cell_props_kernel(const __grid_constant__ GridArgs<N> a) {
    const int med = blockIdx.y;
    const MediumFields &F = a.m[med];
    const GridScalars &s = a.s;
    const GridFluid<N> &g = a.g;
    const long n = s.cells;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int label = F.label[c];
        double x[N], y[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            x[i] = F.x[(long)i * n + c];
            y[i] = F.y[(long)i * n + c];
        }
        const double Po = F.P[n + c];
        const double Sw = F.sat[c], So = F.sat[n + c], Sg = F.sat[2 * n + c];
        // interfacial tension from the previous densities (CalcIFT, compsim/Do_Cycle.cpp:2438-2455)
        double bift;
        if (label == 0) {
            double ro = F.rho[c], rg = F.rho[n + c], ps = 0;
#pragma unroll
            for (int i = 0; i < N; i++) ps += g.parachor[i] * (x[i] * ro - y[i] * rg);
            bift = pow(ps * 1e-6, 3.88);
        } else {
            bift = kIftBase;
        }
        // relative permeabilities and capillary pressures
        double kr0, kr1, kr2, d0, d1, d2, d3, d4, pcw, pcg;
        if (med == 0) {  // CalcSatFs, compsim/Do_Cycle.cpp:161-255
            TableHit hw = table_lookup(s.swt, s.nswt, Sw);
            TableHit hg = table_lookup(s.sgt, s.nsgt, Sg);
            kr0 = hw.kr;
            pcw = hw.pc;
            d0 = hw.dkr;
            kr2 = hg.kr;
            pcg = hg.pc;
            d3 = hg.dkr;
            d4 = 0;
            const double kro0 = s.swt[2], sw0 = s.swt[0];
            double AA = kr0 + hw.krx / kro0, BB = kr2 + hg.krx / kro0;
            double dAA = d0 + hw.dkrx / kro0, dBB = d3 + hg.dkrx / kro0;
            kr1 = kro0 * (AA * BB - kr0 - kr2);
            d1 = kro0 * (dAA * BB - d0);
            d2 = kro0 * (AA * dBB - d3);
            if (bift < kMiscibleIft) {
                double Fi = pow(bift / kIftBase, 1.0 / kIftPower);
                kr1 = Fi * kr1 + (1 - Fi) * So * (1 - sw0);
                kr2 = Fi * kr2 + (1 - Fi) * Sg * (1 - sw0);
                d3 = Fi * d3 + (1 - Fi) * (1 - sw0);
                d1 *= Fi;
                d2 *= Fi;
                d4 = (1 - Fi) * (1 - sw0);
            }
            if (kr1 < 0) kr1 = 0;
            if (kr1 > 1) kr1 = 1;
            if (d1 > 0) d1 = 0;
            if (d2 > 0) d2 = 0;
        } else {  // fCalcSatFs, compsim/Do_Cycle.cpp:420-432
            kr0 = Sw;
            kr1 = So;
            kr2 = Sg;
            d0 = 1;
            d1 = 0;
            d2 = 0;
            d3 = 1;
            d4 = 1;
            pcw = 0;
            pcg = 0;
        }
        // phase pressures (Calc_Phase_P / fCalc_Phase_P, compsim/Do_Cycle.cpp:1418-1443)
        double Pw, Pg;
        if (med == 0) {
            Pw = Po - pcw;
            Pg = (bift < kMiscibleIft) ? Po + pcg * bift / kIftBase : Po + pcg;
        } else {
            Pw = Po;
            Pg = Po;
        }
        // densities, derivatives, viscosities (Calc_Visco)
        double rho_o, rho_g, mu_o, mu_g, dEo[N + 1], dEg[N + 1];
        phase_density_visc<N>(g, x, Po, false, rho_o, mu_o, dEo);
        phase_density_visc<N>(g, y, Pg, true, rho_g, mu_g, dEg);
        // accumulation at the linearisation point (Pre_Mul, compsim/Do_Time_Step.cpp:54-68)
        const double dp = Po - s.refp;
        const double porpor = F.por[c] * (1 + s.cpor * dp + s.dcpor * dp * dp);
#pragma unroll
        for (int i = 0; i < N - 1; i++) F.pre[(long)i * n + c] = porpor * (x[i] * rho_o * So + y[i] * rho_g * Sg);
        F.pre[(long)(N - 1) * n + c] = porpor * (rho_o * So + rho_g * Sg);
        F.pre[(long)N * n + c] = porpor * s.wat_ro * kWatMRo * Sw;
        // diffusion coefficients
        double Do[N], Dg[N];
        phase_diffusion<N>(g, s, x, rho_o, Do);
        phase_diffusion<N>(g, s, y, rho_g, Dg);
        // phase gravity (CalcPhaseGrav, compsim/Do_Cycle.cpp:2022-2037)
        double mwl = 0, mwg = 0;
#pragma unroll
        for (int i = 0; i < N; i++) {
            mwl += x[i] * g.mw[i];
            mwg += y[i] * g.mw[i];
        }
        F.P[c] = Pw;
        F.P[2 * n + c] = Pg;
        F.ift[c] = bift;
        F.kr[c] = kr0;
        F.kr[n + c] = kr1;
        F.kr[2 * n + c] = kr2;
        F.dkr[c] = d0;
        F.dkr[n + c] = d1;
        F.dkr[2 * n + c] = d2;
        F.dkr[3 * n + c] = d3;
        F.dkr[4 * n + c] = d4;
        F.pc[c] = pcw;
        F.pc[n + c] = pcg;
        F.rho[c] = rho_o;
        F.rho[n + c] = rho_g;
        F.mu[c] = mu_o;
        F.mu[n + c] = mu_g;
        F.gam[c] = kGAccG * rho_o * mwl;
        F.gam[n + c] = kGAccG * rho_g * mwg;
#pragma unroll
        for (int k = 0; k <= N; k++) {
            F.dE[(long)(2 * k) * n + c] = dEo[k];
            F.dE[(long)(2 * k + 1) * n + c] = dEg[k];
        }
#pragma unroll
        for (int j = 0; j < N; j++) {
            F.diff[(long)(2 * j) * n + c] = Do[j];
            F.diff[(long)(2 * j + 1) * n + c] = Dg[j];
        }
    }
}

// Upstream-weighted transmissibilities of the +x, +y, +z faces of every cell
// (Calc_Transes, compsim/Do_Cycle.cpp:800-1107; fCalc_Transes :1109-1416).
// trans[t][d] for face direction d: 0/1 oil/gas mobility, 2/3 the same times
// the face-averaged gravity, 4/6 oil d kro/dSw (/ x gravity), 8/9 oil
// d kro/dSg, 10/11 oil d kro/dSo, 5/7 gas d krg/dSg; transS[p][d] = 0 when
// phase p (oil, gas, water) flows out of this cell across the face.
template <int N>
__global__ void __launch_bounds__(128) face_trans_kernel(const __grid_constant__ GridArgs<N> a) {
    const int med = blockIdx.y;
    const MediumFields &F = a.m[med];
    const GridScalars &s = a.s;
    const GridGeom &geo = a.geo;
    const long n = s.cells;
    const double wfac = s.wat_ro * kWatMRo / s.wat_mu;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int ix = (int)(c % s.nx), iy = (int)((c / s.nx) % s.ny), iz = (int)(c / ((long)s.nx * s.ny));
#pragma unroll 1
        for (int d = 0; d < 3; d++) {
            long nb;
            double dl, dn;
            if (d == 0) {
                if (!(s.nx > 1 && ix < s.nx - 1)) continue;
                nb = c + 1;
                dl = geo.di[ix];
                dn = geo.di[ix + 1];
            } else if (d == 1) {
                if (!(s.ny > 1 && iy < s.ny - 1)) continue;
                nb = c + s.nx;
                dl = geo.dj[iy];
                dn = geo.dj[iy + 1];
            } else {
                if (!(s.nz > 1 && iz < s.nz - 1)) continue;
                nb = c + (long)s.nx * s.ny;
                dl = geo.dk[iz];
                dn = geo.dk[iz + 1];
            }
            const double T = F.iftran[(long)d * n + c];
            const double dH = geo.blockH[c] - geo.blockH[nb];
            auto tr = [&](int t, double v) { F.trans[(long)(t * 3 + d) * n + c] = v; };
            auto ts = [&](int p, int v) { F.transS[(long)(p * 3 + d) * n + c] = (signed char)v; };
            // water
            double pot = F.P[c] - F.P[nb] + kGAcc * s.wat_ro * dH;
            long up = pot > 0 ? c : nb;
            if (med == 0) {
                F.wtran[(long)d * n + c] = T * wfac * F.kr[up];
                F.dwtran[(long)d * n + c] = T * wfac * F.dkr[up];
            } else {
                F.wtran[(long)d * n + c] = T * wfac * F.sat[up];
                F.dwtran[(long)d * n + c] = T * wfac;
            }
            ts(2, pot > 0 ? 0 : 1);
            // oil
            {
                const double C1 = F.label[c] == -1 ? 0.0 : 1.0, C2 = F.label[nb] == -1 ? 0.0 : 1.0;
                double mg = (F.gam[c] * dl * C1 + F.gam[nb] * dn * C2) / (C1 * dl + dn * C2);
                if (C1 == 0 && C2 == 0) mg = 0;
                pot = F.P[n + c] - F.P[n + nb] + mg * dH;
                up = pot > 0 ? c : nb;
                // matrix z faces take d kro/dSo of this cell in both directions
                const long up4 = (med == 0 && d == 2) ? c : up;
                double mob = T * (F.rho[c] * dl * C1 + F.rho[nb] * dn * C2) / (F.mu[c] * dl * C1 + F.mu[nb] * dn * C2);
                double k0, k4, k8, k10;
                if (med == 0) {
                    k0 = F.kr[n + up];
                    k4 = F.dkr[n + up];
                    k8 = F.dkr[2 * n + up];
                    k10 = F.dkr[4 * n + up4];
                } else {
                    k0 = F.sat[n + up];
                    k4 = -1;
                    k8 = -1;
                    k10 = 1;
                }
                tr(0, mob * k0);
                tr(2, mg * mob * k0);
                tr(4, mob * k4);
                tr(6, mg * mob * k4);
                tr(8, mob * k8);
                tr(9, mg * mob * k8);
                tr(10, mob * k10);
                tr(11, mg * mob * k10);
                ts(0, pot > 0 ? 0 : 1);
                if (C1 == 0 && C2 == 0) {
                    tr(0, 0); tr(2, 0); tr(4, 0); tr(6, 0); tr(8, 0); tr(9, 0);
                }
            }
            // gas
            {
                const double C1 = F.label[c] == 1 ? 0.0 : 1.0, C2 = F.label[nb] == 1 ? 0.0 : 1.0;
                double mg = (F.gam[n + c] * dl * C1 + F.gam[n + nb] * dn * C2) / (dl * C1 + dn * C2);
                if (C1 == 0 && C2 == 0) mg = 0;
                pot = F.P[2 * n + c] - F.P[2 * n + nb] + mg * dH;
                up = pot > 0 ? c : nb;
                double mob = T * (F.rho[n + c] * dl * C1 + F.rho[n + nb] * dn * C2) /
                             (F.mu[n + c] * dl * C1 + F.mu[n + nb] * dn * C2);
                double k1, k5;
                if (med == 0) {
                    k1 = F.kr[2 * n + up];
                    k5 = F.dkr[3 * n + up];
                } else {
                    k1 = F.sat[2 * n + up];
                    k5 = 1;
                }
                tr(1, mob * k1);
                tr(3, mg * mob * k1);
                tr(5, mob * k5);
                tr(7, mg * mob * k5);
                ts(1, pot > 0 ? 0 : 1);
                if (C1 == 0 && C2 == 0) {
                    tr(1, 0); tr(3, 0); tr(5, 0); tr(7, 0);
                }
            }
        }
    }
}

}  // namespace osr
