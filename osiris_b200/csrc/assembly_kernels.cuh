// Residual of the fully implicit dual-porosity system (FP64, sm_100a).
//
// The reference evaluates its residual row by row (IteratorFunction,
// compsim/Petsc_Functions.cpp:10-1121 for the fracture, 3445-6895 for the
// matrix), recomputing every cell-level term once per row and locating each
// row's cell by a linear search over the row offsets.  Here one thread owns
// one cell of one continuum and writes every row of its block: the per-face
// phase flux factors, the matrix-fracture transfer terms and the well terms
// are formed once and reused by all component rows.
//
// Block layout (PJac, compsim/Init_Calcs.cpp:1013-1116): blocks of all
// matrix cells in cell order, then all fracture cells; a two-phase cell owns
// 2N+4 rows [N fugacity; N-1 component balances; total hydrocarbon; water;
// sum x - 1; sum y - 1; sum S - 1] and a one-phase cell N+3 rows
// [N-1 component balances; total; water; sum w - 1; sum S - 1].  The unknown
// vector uses the same offsets: [x | y, P/PCoeff, Sw, So, Sg] for a
// two-phase cell, [w, P/PCoeff, Sw, S_present] for a one-phase cell
// (UpdateAll/InitGuess2, compsim/PetscAUX.cpp:176-498, 878-964).
#pragma once

// Resident 128-thread CTAs per SM the residual kernel is compiled for (bounds
// its registers).
#ifndef OSR_RES_MIN_BLOCKS
#define OSR_RES_MIN_BLOCKS 4
#endif
#include "grid_kernels.cuh"

namespace osr {

constexpr double kSIC = 9.869232667160128e-13;   // SI_C, compsim/Functions.h:207
constexpr double kWellMinP = 7000000;    // WELL_MIN_P, compsim/Functions.h:6
constexpr double kWellMaxP = 14000000;   // WELL_MAX_P, compsim/Functions.h:5
constexpr double kTStepIf = 1e-5;        // TSTEPIF, compsim/Functions.h:265
constexpr double kMinPPP = 5000000;      // MINPPP, compsim/Functions.h:259
constexpr double kMaxPCoeff = 0.01;      // MAX_P_COEFF, compsim/Functions.h:4
constexpr double kPorTiny = 1e-10;       // inactive-cell porosity

// Stream injected by a gas-injection well: the reference's FlashInjection
// (compsim/Init_Calcs.cpp:1161-1378) at the well's pressure and composition.
struct WellStream {
    double xo[OSR_MAX_NC], yg[OSR_MAX_NC];
    double of, gf;   // oil / gas phase fractions
    double od, gd;   // molar densities
    double ov, gv;   // LBC viscosities
};

struct WellSet {
    int n;
    const int *wi;        // [n][5] type, ix, iy, k0, k1
    const double *wf;     // [n][nc+6]
    const double *re;     // [n] Peaceman radius of the matrix completion (Calc_Re)
    const unsigned char *cond;  // [n] WellCondition latch
    const WellStream *ws; // [n]
    // [n][2][kWellSums] layer sums of the rate split given by the caller (a
    // z-slab run: the sums over the whole reservoir); null: summed here
    const double *sums = nullptr;
};

// Layer sums per well and completion continuum (well_sums_kernel): the sums
// over the own continuum's and the other continuum's completed layers, then
// type 6's mobility-fraction sums SSw, SSo, SSg.
constexpr int kWellSums = 5;

struct AsmScalars {
    double dt, sim_time, pcoeff;
    // per-pass controls in device memory ([dt, time, PCoeff]) read in place
    // of the three values above when set (a Newton step replayed as a graph)
    const double *ctl;
    double sf1, sf3;      // ShapeFactor_1 / _3 without the geometric sums' zero gate applied
    double sigma, lf, re_f;
    int diff_off;         // CDIF present with a zero value: both diffusive shape factors vanish
};

template <int N>
struct AsmArgs {
    GridArgs<N> a;
    AsmScalars k;
    WellSet w;
    const double *tor;    // [cells]
    const long *rowoff;   // [2 cells + 1]
    double *f;            // residual
    double *fscale;       // optional: sum of |terms| of each row
};

__device__ __forceinline__ int block_rows(int label, int N) { return label == 0 ? 2 * N + 4 : N + 3; }

// ---------------------------------------------------------------------------
// Injection flash (one thread per well).
// ---------------------------------------------------------------------------
template <int N>
__global__ void well_stream_kernel(const __grid_constant__ GridFluid<N> g, int nw, const int *wi, const double *wf,
                                   WellStream *out) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nw) return;
    const int type = wi[w * 5];
    WellStream s;
    for (int i = 0; i < OSR_MAX_NC; i++) s.xo[i] = s.yg[i] = 0;
    s.of = s.gf = s.od = s.gd = s.ov = s.gv = 0;
    if (type != 3 && type != 8) {
        out[w] = s;
        return;
    }
    const double *row = wf + (long)w * (N + 6);
    const double Pin = type == 3 ? row[0] : row[1];
    double z[N], K[N], xo[N], yg[N];
    const FluidTable<N> &f = g.f;
    const double T = g.T;
    for (int i = 0; i < N; i++) {
        z[i] = row[4 + i];
        K[i] = (f.pc[i] / Pin) * exp(f.wil[i] * (1 - f.tc[i] / T));
        xo[i] = yg[i] = 0;
    }
    const double rt = kR * T;
    double L = 0, Lb = 10, Zl = 1, Zg = 1, esum = 0;
    int k = 0;
    do {
        L = 0.6;
        int j = 0;
        double step;
        do {
            double F = 0, dF = 0;
            for (int i = 0; i < N; i++) {
                double t = K[i] >= 0 ? (1 - K[i]) / (L + (1 - L) * K[i]) : 1 / (L - 1);
                F += z[i] * t;
                dF -= z[i] * t * t;
            }
            step = F / dF;
            L -= step;
            j++;
        } while (step * step > kRRTol && j < kRRMaxIt);
        if (L > 1) L = 1;
        else if (L < 0) L = 0;
        esum = fabs(Lb - L);
        Lb = L;
        for (int i = 0; i < N; i++) {
            if (K[i] >= 0) {
                xo[i] = z[i] / (L + K[i] * (1 - L));
                yg[i] = K[i] * xo[i];
            } else {
                xo[i] = 0;
                yg[i] = yg[i] / (1 - L);
            }
        }
        double Al = 0, Bl = 0, Ag = 0, Bg = 0;
        for (int i = 0; i < N; i++) {
            Bl += xo[i] * f.b[i];
            Bg += yg[i] * f.b[i];
            for (int jj = 0; jj < N; jj++) {
                double t = g.sa[i] * g.sa[jj] * f.bic[i * N + jj];
                Al += xo[i] * xo[jj] * t;
                Ag += yg[i] * yg[jj] * t;
            }
        }
        const double Cal = Al, Cbl = Bl, Cag = Ag, Cbg = Bg;
        Al *= Pin / (rt * rt);
        Bl *= Pin / rt;
        Ag *= Pin / (rt * rt);
        Bg *= Pin / rt;
        const bool srk = f.srk != 0;
        const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
        Zl = phase_z(Al, Bl, srk, false);
        Zg = phase_z(Ag, Bg, srk, true);
        for (int i = 0; i < N; i++) {
            double tl = 0, tg = 0;
            for (int jj = 0; jj < N; jj++) {
                double t = g.sa[i] * g.sa[jj] * f.bic[i * N + jj];
                tl += xo[jj] * t;
                tg += yg[jj] * t;
            }
            double t1l = f.b[i] / Cbl, t1g = f.b[i] / Cbg;
            double EEl = 2 * tl / Cal - t1l, EEg = 2 * tg / Cag - t1g;
            double DDl = Al / (Bl * (d1 - d2)), DDg = Ag / (Bg * (d1 - d2));
            double FFl = log((Zl + d2 * Bl) / (Zl + d1 * Bl)), FFg = log((Zg + d2 * Bg) / (Zg + d1 * Bg));
            double phiL = exp(t1l * (Zl - 1) - log(Zl - Bl) + DDl * EEl * FFl);
            double phiG = exp(t1g * (Zg - 1) - log(Zg - Bg) + DDg * EEg * FFg);
            double fL = xo[i] * phiL, fG = yg[i] * phiG;
            if (z[i] != 0) {
                if (fG != 0) K[i] *= fL / fG;
                else K[i] = -1;
                if (fL != fL) K[i] = -1;
                if (fG != fG) K[i] = 1;
            }
        }
        k++;
    } while (esum > kSSTol && k < kSSMaxIt);
    if (fabs(L) < kLZero) {
        s.of = 0;
        s.gf = 1;
    } else if (fabs(1 - L) < kLZero) {
        s.of = 1;
        s.gf = 0;
    } else {
        s.of = L;
        s.gf = 1 - L;
    }
    s.od = Pin / (Zl * rt);
    s.gd = Pin / (Zg * rt);
    for (int ph = 0; ph < 2; ph++) {
        const double *w = ph ? yg : xo;
        double s1 = 0, s2 = 0, ro = 0, tcm = 0, pcm = 0, mwm = 0;
        for (int n = 0; n < N; n++) {
            double t = w[n] * g.smw[n];
            s1 += t * g.mui[n];
            s2 += t;
            ro += w[n] * g.vcm[n];
            tcm += w[n] * f.tc[n];
            pcm += w[n] * g.pcr_atm[n];
            mwm += w[n] * g.mw[n];
        }
        double Er = (ph ? s.gd : s.od) * ro;
        double eta = pow(tcm, 1.0 / 6) / (sqrt(mwm) * pow(pcm, 2.0 / 3));
        double r1 = 0.10230 + 0.023364 * Er + 0.058533 * Er * Er - 0.040758 * Er * Er * Er + 0.0093324 * Er * Er * Er * Er;
        double mu = s1 / s2 + (r1 * r1 * r1 * r1 - 1e-4) / eta;
        if (ph) s.gv = mu;
        else s.ov = mu;
    }
    for (int i = 0; i < N; i++) {
        s.xo[i] = xo[i];
        s.yg[i] = yg[i];
    }
    out[w] = s;
}

// ---------------------------------------------------------------------------
// Row layout and unknown maps.
// ---------------------------------------------------------------------------

// Block sizes of every cell of both continua (matrix first); an exclusive
// scan turns them into the row offsets.
static __global__ void block_size_kernel(const signed char *lab_m, const signed char *lab_f, long cells, int N, long *sizes) {
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < 2 * cells; b += (long)gridDim.x * blockDim.x) {
        const signed char l = b < cells ? lab_m[b] : lab_f[b - cells];
        sizes[b] = block_rows(l, N);
    }
}

// Exclusive scan of the block sizes into the row offsets (2 cells + 1
// outputs), across the whole GPU in three launches: every CTA sums its
// contiguous chunk of sizes (coalesced, strided by the CTA's threads); one
// warp scans the kScanBlocks chunk sums into chunk bases (and the total);
// every CTA then scans its chunk in tiles of kScanThreads with warp shuffles,
// carrying the running sum from tile to tile.  Integer sums: exact and
// independent of the launch shape.
constexpr int kScanBlocks = 296;
constexpr int kScanThreads = 256;

__device__ __forceinline__ long scan_chunk_begin(long nb, int blk) {
    const long chunk = (nb + kScanBlocks - 1) / kScanBlocks;
    const long b = (long)blk * chunk;
    return b < nb ? b : nb;
}

static __global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(const long *sizes, long nb, long *part) {
    __shared__ long warp_sum[kScanThreads / 32];
    const long b0 = scan_chunk_begin(nb, blockIdx.x), b1 = scan_chunk_begin(nb, blockIdx.x + 1);
    long s = 0;
    for (long b = b0 + threadIdx.x; b < b1; b += kScanThreads) s += sizes[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long t = 0;
        for (int w = 0; w < kScanThreads / 32; w++) t += warp_sum[w];
        part[blockIdx.x] = t;
    }
}

// one warp: exclusive scan of the chunk sums in place, total into off[nb]
static __global__ void scan_bases_kernel(long *part, long nb, long *off) {
    const int lane = threadIdx.x;
    long carry = 0;
    for (int i0 = 0; i0 < kScanBlocks; i0 += 32) {
        const int i = i0 + lane;
        const long v = i < kScanBlocks ? part[i] : 0;
        long incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (i < kScanBlocks) part[i] = carry + incl - v;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) off[nb] = carry;
}

static __global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const long *sizes, long nb, const long *base,
                                                                       long *off) {
    __shared__ long warp_tot[kScanThreads / 32];
    __shared__ long tile_total;
    const long b0 = scan_chunk_begin(nb, blockIdx.x), b1 = scan_chunk_begin(nb, blockIdx.x + 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long carry = base[blockIdx.x];
    for (long t0 = b0; t0 < b1; t0 += kScanThreads) {
        const long b = t0 + threadIdx.x;
        const long v = b < b1 ? sizes[b] : 0;
        long incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        long before = 0, total = 0;
        for (int w = 0; w < kScanThreads / 32; w++) {
            if (w < warp) before += warp_tot[w];
            total += warp_tot[w];
        }
        if (b < b1) off[b] = carry + before + incl - v;
        if (threadIdx.x == 0) tile_total = total;
        __syncthreads();
        carry += tile_total;
        __syncthreads();
    }
}

// Largest oil pressure over both continua (CalcPCoeff,
// compsim/Init_Calcs.cpp:1118-1130), as an ordered-integer atomic max of
// non-negative doubles.
static __global__ void pcoeff_kernel(const double *Pm, const double *Pf, long cells, unsigned long long *out) {
    unsigned long long best = 0;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += (long)gridDim.x * blockDim.x) {
        double a = Pm[c], b = Pf[c];
        double v = a > b ? a : b;
        if (v > 0) {
            unsigned long long u = (unsigned long long)__double_as_longlong(v);
            if (u > best) best = u;
        }
    }
    for (int o = 16; o; o >>= 1) {
        unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        if (v > best) best = v;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

// State -> unknowns (InitGuess2).
template <int N>
__global__ void init_guess_kernel(const __grid_constant__ GridArgs<N> a, const long *rowoff, double pcoeff_arg,
                                  const double *ctl, double *x) {
    const double pcoeff = ctl ? ctl[2] : pcoeff_arg;
    const long n = a.s.cells;
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < 2 * n; b += (long)gridDim.x * blockDim.x) {
        const int med = b >= n;
        const long c = med ? b - n : b;
        const MediumFields &F = a.m[med];
        double *o = x + rowoff[b];
        const signed char l = F.label[c];
        if (l == 0) {
            for (int i = 0; i < N; i++) o[i] = F.x[(long)i * n + c];
            for (int i = 0; i < N; i++) o[N + i] = F.y[(long)i * n + c];
            o[2 * N] = F.P[n + c] / pcoeff;
            o[2 * N + 1] = F.sat[c];
            o[2 * N + 2] = F.sat[n + c];
            o[2 * N + 3] = F.sat[2 * n + c];
        } else {
            const double *w = l == 1 ? F.x : F.y;
            for (int i = 0; i < N; i++) o[i] = w[(long)i * n + c];
            o[N] = F.P[n + c] / pcoeff;
            o[N + 1] = F.sat[c];
            o[N + 2] = F.sat[(l == 1 ? 1 : 2) * n + c];
        }
    }
}

// Unknowns -> state, without the phase control of a full step (UpdateAll's
// unpacking, compsim/PetscAUX.cpp:206-478): compositions clamped to [0, 1]
// and renormalised (uniform when they sum to zero), the oil pressure limited
// by the reference's step rule and floored at MINPPP, saturations clamped
// and renormalised.
template <int N>
__global__ void update_all_kernel(const __grid_constant__ GridArgs<N> a, const long *rowoff, double pcoeff_arg,
                                  const double *ctl, const double *x) {
    const double pcoeff = ctl ? ctl[2] : pcoeff_arg;
    const long n = a.s.cells;
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < 2 * n; b += (long)gridDim.x * blockDim.x) {
        const int med = b >= n;
        const long c = med ? b - n : b;
        const MediumFields &F = a.m[med];
        const double *o = x + rowoff[b];
        const signed char l = F.label[c];
        auto unpack_w = [&](double *w, const double *src) {
            double s = 0;
            double v[N];
            for (int i = 0; i < N; i++) {
                double t = src[i];
                if (t < 0) t = 0;   // EPS_COMP = 0
                else if (t > 1) t = 1;
                v[i] = t;
                s += t;
            }
            for (int i = 0; i < N; i++) w[(long)i * n + c] = s != 0 ? v[i] / s : 1.0 / N;
        };
        auto unpack_p = [&](double xv) {
            double Pold = F.P[n + c];
            double Pn;
            if (fabs(pcoeff * xv) > Pold * (1 + kMaxPCoeff)) {
                double d = xv * pcoeff - Pold;
                Pn = Pold + kMaxPCoeff * (d > 0 ? 1.0 : (d < 0 ? -1.0 : 0.0));
            } else {
                Pn = xv * pcoeff;
            }
            if (Pn < kMinPPP) Pn = kMinPPP;
            F.P[n + c] = Pn;
        };
        auto clamp01 = [](double v) { return v < 0 ? 0.0 : (v > 1 ? 1.0 : v); };
        if (l == 0) {
            unpack_w(F.x, o);
            unpack_w(F.y, o + N);
            unpack_p(o[2 * N]);
            double sw = clamp01(o[2 * N + 1]), so = clamp01(o[2 * N + 2]), sg = clamp01(o[2 * N + 3]);
            double s = sw + so + sg;
            if (s != 0) {
                sw /= s;
                so /= s;
                sg /= s;
            }
            F.sat[c] = sw;
            F.sat[n + c] = so;
            F.sat[2 * n + c] = sg;
        } else {
            unpack_w(l == 1 ? F.x : F.y, o);
            unpack_p(o[N]);
            double sw = o[N + 1], sh = o[N + 2];
            if (sw < 0) sw = 0;
            if (sw > 1) sw = 1;
            if (sh > 1) sh = 1;
            if (sh < 0) sh = 0;
            double s = sw + sh;
            if (s != 0) {
                sw /= s;
                sh /= s;
            }
            F.sat[c] = sw;
            F.sat[(l == 1 ? 1 : 2) * n + c] = sh;
        }
    }
}

// ---------------------------------------------------------------------------
// Residual.
// ---------------------------------------------------------------------------

// Well rates of one completion cell (the "Wells&Commons" regions of
// IteratorFunction, compsim/Petsc_Functions.cpp:164-702 for the fracture and
// 3505-4044 for the matrix).  own/oth are the completion's and the other
// continuum's fields; returns the index of the last injection well that set
// the component stream, or -1.
struct WellRates {
    double Qw, Qo, Qg, PIw, PIo, PIg;
    int iwell;
};

template <int N>
__device__ void well_rates(const AsmArgs<N> &A, int med, long c, int ix, int iy, int iz, WellRates &r) {
    const GridScalars &s = A.a.s;
    const MediumFields &O = A.a.m[med], &X = A.a.m[1 - med];
    const long n = s.cells;
    const double *dk = A.a.geo.dk;
    const double watRo = s.wat_ro, watMu = s.wat_mu;
    const double wfac = watRo * kWatMRo;
    r = WellRates{0, 0, 0, 0, 0, 0, -1};
    const double t = A.k.ctl ? A.k.ctl[1] : A.k.sim_time;
    // own-cell quantities
    const double Pw = O.P[c], Po = O.P[n + c], Pg = O.P[2 * n + c];
    const double krw = O.kr[c], kro = O.kr[n + c], krg = O.kr[2 * n + c];
    const double rho_o = O.rho[c], rho_g = O.rho[n + c], mu_o = O.mu[c], mu_g = O.mu[n + c];
    const double sqk = sqrt(O.perm[n + c] * O.perm[c]);
    const double sgt_kr = s.sgt[(s.nsgt - 1) * 4 + 1];
    for (int i = 0; i < A.w.n; i++) {
        const int *wi = A.w.wi + 5 * i;
        if (!(ix == wi[1] && iy == wi[2] && iz >= wi[3] && iz <= wi[4])) continue;
        const double *wf = A.w.wf + (long)i * (N + 6);
        const int type = wi[0];
        const double rw = wf[3], skin = wf[2];
        double Re = med == 0 ? A.w.re[i] : A.k.re_f;
        // completion factor log term of this continuum and of the other one
        auto own_log = [&](double re) { return med == 0 ? log(re / rw) + skin : log((rw + A.k.re_f) / rw) + skin; };
        auto oth_log = [&](double re) { return med == 0 ? log((rw + A.k.re_f) / rw) + skin : log(re / rw) + skin; };
        const bool late = type == 3 || type == 8;
        const double t0 = late ? wf[N + 4] : wf[4], t1 = late ? wf[N + 5] : wf[5];
        const bool active = (fabs(t - t0) <= kTStepIf) || (fabs(t - t1) <= kTStepIf) || (t >= t0 && t <= t1);
        if (!active) continue;
        const bool cond = A.w.cond[i] != 0;
        // sums over the completed layers of both continua
        auto layer_sum = [&](auto &&term) {
            double acc = 0;
            for (int j = wi[3]; j <= wi[4]; j++) {
                const long cj = ix + (long)s.nx * (iy + (long)s.ny * j);
                double S2 = dk[j] * sqrt(O.perm[cj] * O.perm[n + cj]) / own_log(Re);
                acc += term(O, cj, S2);
                S2 = dk[j] * sqrt(X.perm[cj] * X.perm[n + cj]) / oth_log(Re);
                acc += term(X, cj, S2);
            }
            return acc;
        };
        // the caller's layer sums of this well and completion continuum, if any
        const double *wsum = A.w.sums ? A.w.sums + ((long)i * 2 + med) * kWellSums : nullptr;
        auto S1_2pi = [&]() { return 2 * kSIC * kPi * dk[iz] * sqk / own_log(Re); };
        auto S1_plain = [&]() { return dk[iz] * sqrt(O.perm[c] * O.perm[n + c]) / own_log(Re); };
        auto all_pi = [&](double S1) {
            r.PIw = S1 * wfac * krw / watMu;
            r.PIo = S1 * rho_o * kro / mu_o;
            r.PIg = S1 * rho_g * krg / mu_g;
            r.Qw = r.PIw * (wf[0] - Pw);
            r.Qo = r.PIo * (wf[0] - Po);
            r.Qg = r.PIg * (wf[0] - Pg);
        };
        auto producer_signs = [&]() {
            if (r.Qw > 0 || (r.Qw - r.Qw) != 0) { r.Qw = 0; r.PIw = 0; }
            if (r.Qo > 0 || (r.Qo - r.Qo) != 0) { r.Qo = 0; r.PIo = 0; }
            if (r.Qg > 0 || (r.Qg - r.Qg) != 0) { r.Qg = 0; r.PIg = 0; }
        };
        if (type == 0) {  // constant bottom-hole pressure, production
            if (med == 0 && Re <= rw) Re += rw;
            all_pi(S1_2pi());
            if (Po < kWellMinP) {
                r.Qw = r.Qo = r.Qg = 0;
                r.PIw = r.PIo = r.PIg = 0;
            } else if (wf[1] != 0 && (-r.Qo) > wf[1]) {
                r.Qo = -wf[1];
                r.Qw = r.Qo * krw * wfac * mu_o / (kro * rho_o * watMu);
                r.Qg = r.Qo * krg * rho_g * mu_o / (kro * rho_o * mu_g);
                r.PIw = r.PIo = r.PIg = 0;
            }
            producer_signs();
        } else if (type == 1) {  // constant bottom-hole pressure, gas production
            all_pi(S1_2pi());
            producer_signs();
            if (cond) {
                double SS = wsum ? wsum[0] / O.mu[n + c] + wsum[1] / X.mu[n + c]
                                 : layer_sum([&](const MediumFields &M, long cj, double S2) {
                                       return M.rho[n + cj] * S2 * M.kr[2 * n + cj] / M.mu[n + c];
                                   });
                double S1 = S1_plain();
                if (SS != 0) r.Qg = -S1 * wf[1] * rho_g * krg / (mu_g * SS);
                r.Qw = r.Qg * krw * wfac * mu_g / (krg * rho_g * watMu);
                r.Qo = r.Qg * kro * rho_o * mu_g / (krg * rho_g * mu_o);
            }
        } else if (type == 2) {  // constant bottom-hole pressure, water injection
            double S1 = S1_2pi();
            r.PIw = S1 * wfac * krw / watMu;
            r.Qw = r.PIw * (wf[0] - Pw);
            if (r.Qw < 0 || (r.Qw - r.Qw) != 0) { r.Qw = 0; r.PIw = 0; }
            if (cond) {
                double SS = wsum ? wsum[0] + wsum[1] : layer_sum([&](const MediumFields &M, long cj, double S2) {
                    return watRo * S2 * M.kr[cj] / watMu;
                });
                S1 = S1_plain();
                if (SS != 0) r.Qw = S1 * wf[1] * wfac * krw / (watMu * SS);
            }
        } else if (type == 3) {  // constant bottom-hole pressure, gas injection
            const WellStream &ws = A.w.ws[i];
            if (med == 0 && Re <= rw) Re += rw;
            double S1 = S1_2pi();
            r.PIg = S1 * ws.gd * sgt_kr * ws.gf / ws.gv;
            r.Qg = r.PIg * (wf[0] - Pg);
            r.PIo = r.PIg * ws.of / ws.gf;
            r.Qo = r.PIo * (wf[0] - Pg);
            if (r.Qo < 0 || (r.Qo - r.Qo) != 0) { r.Qo = 0; r.PIo = 0; }
            if (r.Qg < 0 || (r.Qg - r.Qg) != 0) { r.Qg = 0; r.PIg = 0; }
            r.iwell = i;
            if (cond) {
                double SS = wsum ? wsum[0] + wsum[1]
                                 : layer_sum([&](const MediumFields &, long, double S2) { return S2; });
                S1 = S1_plain();
                if (SS != 0) r.Qg = S1 * wf[1] / SS;
                if (SS != 0) r.Qo = r.Qg * ws.of / ws.gf;
            }
        } else if (type == 4 || type == 5 || type == 6) {  // constant oil / gas / total rate
            double SS, S1 = S1_plain();
            if (type == 6 && wsum) {
                SS = wsum[0] / O.mu[c] + wsum[1] / X.mu[c];
                const double QoP = wsum[3] * wf[0] / (wsum[2] + wsum[3] + wsum[4]);
                if (SS != 0) r.Qo = -S1 * QoP * rho_o * kro / (mu_o * SS);
            } else if (type == 6) {
                double SSw = 0, SSo = 0, SSg = 0;
                SS = 0;
                for (int j = wi[3]; j <= wi[4]; j++) {
                    const long cj = ix + (long)s.nx * (iy + (long)s.ny * j);
                    for (int pass = 0; pass < 2; pass++) {
                        const MediumFields &M = pass ? X : O;
                        double mob = (M.kr[cj] / watMu) + (M.kr[n + cj] / M.mu[cj]) + (M.kr[2 * n + cj] / M.mu[n + cj]);
                        SSw += (M.kr[cj] / watMu) / mob;
                        SSo += (M.kr[n + cj] / M.mu[cj]) / mob;
                        SSg += (M.kr[2 * n + cj] / M.mu[n + cj]) / mob;
                        double S2 = dk[j] * sqrt(M.perm[cj] * M.perm[n + cj]) / (pass ? oth_log(Re) : own_log(Re));
                        SS += M.rho[cj] * S2 * M.kr[n + cj] / M.mu[c];
                    }
                }
                const double QoP = SSo * wf[0] / (SSw + SSo + SSg);
                if (SS != 0) r.Qo = -S1 * QoP * rho_o * kro / (mu_o * SS);
            } else if (type == 4) {
                SS = wsum ? wsum[0] / O.mu[c] + wsum[1] / X.mu[c]
                          : layer_sum([&](const MediumFields &M, long cj, double S2) {
                                return M.rho[cj] * S2 * M.kr[n + cj] / M.mu[c];
                            });
                if (SS != 0) r.Qo = -S1 * wf[0] * rho_o * kro / (mu_o * SS);
            } else {
                SS = wsum ? wsum[0] / O.mu[n + c] + wsum[1] / X.mu[n + c]
                          : layer_sum([&](const MediumFields &M, long cj, double S2) {
                                return M.rho[n + cj] * S2 * M.kr[2 * n + cj] / M.mu[n + c];
                            });
                if (SS != 0) r.Qg = -S1 * wf[1] * rho_g * krg / (mu_g * SS);
            }
            if (type == 5) {
                r.Qw = r.Qg * krw * wfac * mu_g / (krg * rho_g * watMu);
                r.Qo = r.Qg * kro * rho_o * mu_g / (krg * rho_g * mu_o);
            } else {
                r.Qw = r.Qo * krw * wfac * mu_o / (kro * rho_o * watMu);
                r.Qg = r.Qo * krg * rho_g * mu_o / (kro * rho_o * mu_g);
            }
            if (cond) {
                all_pi(S1_2pi());
                producer_signs();
            }
            if (type == 4 && med == 1 && Po < kWellMinP) {
                r.Qw = r.Qo = r.Qg = 0;
                r.PIw = r.PIo = r.PIg = 0;
            }
        } else if (type == 7) {  // constant water injection rate: zero unless latched
            if (cond) {
                double S1 = S1_2pi();
                r.PIw = S1 * wfac * krw / watMu;
                r.Qw = r.PIw * (wf[0] - Pw);
                if (r.Qw < 0 || (r.Qw - r.Qw) != 0) { r.Qw = 0; r.PIw = 0; }
            }
        } else if (type == 8) {  // constant gas injection rate
            const WellStream &ws = A.w.ws[i];
            if (med == 0 && Re <= rw) Re += rw;
            double SS = wsum ? wsum[0] + wsum[1]
                             : layer_sum([&](const MediumFields &, long, double S2) { return S2; });
            double S1 = S1_plain();
            if (SS != 0) r.Qg = S1 * wf[0] / SS;
            if (SS != 0) r.Qo = r.Qg * ws.of / ws.gf;
            if (med == 1) S1 = S1_2pi();
            if (cond) {
                r.PIg = S1 * ws.gd * sgt_kr * ws.gf / ws.gv;
                r.Qg = r.PIg * (wf[1] - Pg);
                r.PIo = r.PIg * ws.of / ws.gf;
                r.Qo = r.PIo * (wf[1] - Pg);
                if (r.Qo < 0 || (r.Qo - r.Qo) != 0) { r.Qo = 0; r.PIo = 0; }
                if (r.Qg < 0 || (r.Qg - r.Qg) != 0) { r.Qg = 0; r.PIg = 0; }
            }
            if (Po > kWellMaxP) {
                r.Qw = r.Qo = r.Qg = 0;
                r.PIw = r.PIo = r.PIg = 0;
            }
            r.iwell = i;
        }
    }
}

// Layer sums of the rate split of every well and completion continuum over
// the layers [l0, l1) of this grid (the layer_sum terms of well_rates without
// the completion cell's viscosity, which well_rates divides by; the own and
// the other continuum summed apart): sums[w][med][kWellSums].  A z-slab run
// takes them over each rank's owned layers and adds them over the ranks.
template <int N>
__global__ void well_sums_kernel(const __grid_constant__ AsmArgs<N> A, int l0, int l1, double *sums) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * A.w.n) return;
    const int i = t >> 1, med = t & 1;
    const GridScalars &s = A.a.s;
    const MediumFields &O = A.a.m[med], &X = A.a.m[1 - med];
    const long n = s.cells;
    const double *dk = A.a.geo.dk;
    const int *wi = A.w.wi + 5 * i;
    const double *wf = A.w.wf + (long)i * (N + 6);
    const int type = wi[0], ix = wi[1], iy = wi[2];
    const double rw = wf[3], skin = wf[2];
    double Re = med == 0 ? A.w.re[i] : A.k.re_f;
    if ((type == 3 || type == 8) && med == 0 && Re <= rw) Re += rw;
    const double own_l = med == 0 ? log(Re / rw) + skin : log((rw + A.k.re_f) / rw) + skin;
    const double oth_l = med == 0 ? log((rw + A.k.re_f) / rw) + skin : log(Re / rw) + skin;
    const double watRo = s.wat_ro, watMu = s.wat_mu;
    double acc[kWellSums] = {0, 0, 0, 0, 0};
    const int j0 = wi[3] > l0 ? wi[3] : l0, j1 = wi[4] < l1 - 1 ? wi[4] : l1 - 1;
    for (int j = j0; j <= j1; j++) {
        const long cj = ix + (long)s.nx * (iy + (long)s.ny * j);
        for (int pass = 0; pass < 2; pass++) {
            const MediumFields &M = pass ? X : O;
            const double S2 = dk[j] * sqrt(M.perm[cj] * M.perm[n + cj]) / (pass ? oth_l : own_l);
            double term = 0;
            if (type == 1 || type == 5) term = M.rho[n + cj] * S2 * M.kr[2 * n + cj];
            else if (type == 2) term = watRo * S2 * M.kr[cj] / watMu;
            else if (type == 3 || type == 8) term = S2;
            else if (type == 4 || type == 6) term = M.rho[cj] * S2 * M.kr[n + cj];
            acc[pass] += term;
            if (type == 6) {
                const double mob = (M.kr[cj] / watMu) + (M.kr[n + cj] / M.mu[cj]) + (M.kr[2 * n + cj] / M.mu[n + cj]);
                acc[2] += (M.kr[cj] / watMu) / mob;
                acc[3] += (M.kr[n + cj] / M.mu[cj]) / mob;
                acc[4] += (M.kr[2 * n + cj] / M.mu[n + cj]) / mob;
            }
        }
    }
    for (int q = 0; q < kWellSums; q++) sums[(long)t * kWellSums + q] = acc[q];
}

// Well rates and productivity indices of every cell-medium at the current
// state ([2 cells][3] water, oil, gas) and the injection well setting each
// completion's component split (-1 when none).
template <int N>
__global__ void well_terms_kernel(const __grid_constant__ AsmArgs<N> A, double *q, double *pi, int *iw) {
    const GridScalars &s = A.a.s;
    const long n = s.cells;
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < 2 * n; b += (long)gridDim.x * blockDim.x) {
        const int med = b >= n;
        const long c = med ? b - n : b;
        const int ix = (int)(c % s.nx), iy = (int)((c / s.nx) % s.ny), iz = (int)(c / ((long)s.nx * s.ny));
        WellRates r;
        well_rates<N>(A, med, c, ix, iy, iz, r);
        q[3 * b] = r.Qw;
        q[3 * b + 1] = r.Qo;
        q[3 * b + 2] = r.Qg;
        pi[3 * b] = r.PIw;
        pi[3 * b + 1] = r.PIo;
        pi[3 * b + 2] = r.PIg;
        iw[b] = r.iwell;
    }
}

// Fugacity coefficients of one phase at the phase's own pressure with Z taken
// from the stored density, as the two-phase rows evaluate them
// (compsim/Petsc_Functions.cpp:4559-4621).  The reference recomputes the
// mixing sums for every component row; they do not depend on the row, so they
// are formed once per phase here, with the same operations in the same order
// as the per-row evaluation.  s[k] is the
// k-th attraction row sum sum_j w_j sa_k sa_j (1 - kij), which is also the
// component's own t_i.
template <int N>
struct PhaseFug {
    double s[N];
    double Ca, Cb, Z, DD, FF, lzb;

    __device__ __forceinline__ PhaseFug(const GridFluid<N> &g, const double *w, long n, long c, double P, double rho) {
        const FluidTable<N> &f = g.f;
        const double rt = kR * g.T;
        double wv[N];
#pragma unroll
        for (int k = 0; k < N; k++) wv[k] = w[(long)k * n + c];
        double A = 0, B = 0;
#pragma unroll
        for (int k = 0; k < N; k++) {
            B += wv[k] * f.b[k];
            double sk = 0;
#pragma unroll
            for (int j = 0; j < N; j++) sk += wv[j] * g.sa[k] * g.sa[j] * f.bic[k * N + j];
            s[k] = sk;
            A += wv[k] * sk;
        }
        Ca = A;
        Cb = B;
        A *= P / (rt * rt);
        B *= P / rt;
        Z = P / (rho * rt);
        const bool srk = f.srk != 0;
        const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
        DD = A / (B * (d1 - d2));
        FF = log((Z + d2 * B) / (Z + d1 * B));
        lzb = log(Z - B);
    }

    // fugacity coefficient of component i
    __device__ __forceinline__ double coeff(const FluidTable<N> &f, int i) const {
        const double t1 = f.b[i] / Cb;
        const double EE = 2 * s[i] / Ca - t1;
        return exp(t1 * (Z - 1) - lzb + DD * EE * FF);
    }
};

// One face of a cell: neighbour index, distances, areas.
struct Face {
    long nb;        // neighbour cell
    long tc;        // cell holding the face's transmissibilities (+ faces: this cell; - faces: the neighbour)
    int d;          // direction 0 x, 1 y, 2 z
    double sgn;     // +1 for the + face, -1 for the - face
    double dl, dn;  // block size along d of this cell and of the neighbour
    double area2;   // 2 * cross-section product of the other two block sizes
};

template <int N>
__device__ __forceinline__ int cell_faces(const AsmArgs<N> &A, long c, int ix, int iy, int iz, Face *fc) {
    const GridScalars &s = A.a.s;
    const GridGeom &geo = A.a.geo;
    const long sx = 1, sy = s.nx, sz = (long)s.nx * s.ny;
    int k = 0;
    // order of the reference's intra-continuum diffusion loop: +x, -x, +y, -y, +z, -z
    if (ix < s.nx - 1) fc[k++] = Face{c + sx, c, 0, 1, geo.di[ix], geo.di[ix + 1], 2 * geo.dj[iy] * geo.dk[iz]};
    if (ix > 0) fc[k++] = Face{c - sx, c - sx, 0, -1, geo.di[ix], geo.di[ix - 1], 2 * geo.dj[iy] * geo.dk[iz]};
    if (iy < s.ny - 1) fc[k++] = Face{c + sy, c, 1, 1, geo.dj[iy], geo.dj[iy + 1], 2 * geo.di[ix] * geo.dk[iz]};
    if (iy > 0) fc[k++] = Face{c - sy, c - sy, 1, -1, geo.dj[iy], geo.dj[iy - 1], 2 * geo.di[ix] * geo.dk[iz]};
    if (iz < s.nz - 1) fc[k++] = Face{c + sz, c, 2, 1, geo.dk[iz], geo.dk[iz + 1], 2 * geo.di[ix] * geo.dj[iy]};
    if (iz > 0) fc[k++] = Face{c - sz, c - sz, 2, -1, geo.dk[iz], geo.dk[iz - 1], 2 * geo.di[ix] * geo.dj[iy]};
    return k;
}

__device__ __forceinline__ double porpor_at(const MediumFields &F, const GridScalars &s, long c) {
    const double dp = F.P[s.cells + c] - s.refp;
    return F.por[c] * (1 + s.cpor * dp + s.dcpor * dp * dp);
}

// Threads per CTA of the residual kernel.
constexpr int kResThreads = 128;

// Per-thread face tables of the residual kernel in shared memory, entry e of
// thread t at [e][t] (a warp reads consecutive words): the advective and
// gravity factors and upstream cell of each (phase, face), the diffusion
// factor of each (phase, face), the neighbour of each face, and bits: 1 << q
// a + face, 1 << (6 + q) an inactive neighbour, 1 << (12 + 6 p + q) no
// diffusive flux.  The component rows read these once per row; as a local
// array the thread's frame (about 800 bytes, 512 threads per SM) exceeds L1.
// Cell indices fit 32 bits (the host checks the grid size).
struct ResFaces {
    double kp[12][kResThreads], kg[12][kResThreads], db[12][kResThreads];
    int up[12][kResThreads], nb[6][kResThreads];
    unsigned bits[kResThreads];
};

// SCALE: the row scales (sum of |terms| of each row) are written to A.fscale.
// Launched with kResThreads threads per CTA.
template <int N, bool SCALE>
__global__ void __launch_bounds__(kResThreads, OSR_RES_MIN_BLOCKS) residual_kernel(const __grid_constant__ AsmArgs<N> A) {
    __shared__ ResFaces sf;
    const int t = threadIdx.x;
    const GridScalars &s = A.a.s;
    const GridGeom &geo = A.a.geo;
    const long n = s.cells;
    const double wfac = s.wat_ro * kWatMRo;
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < 2 * n; b += (long)gridDim.x * blockDim.x) {
        const int med = b >= n;
        const long c = med ? b - n : b;
        const MediumFields &F = A.a.m[med];
        const MediumFields &M = A.a.m[0], &Fr = A.a.m[1];
        const long row0 = A.rowoff[b];
        const signed char lab = F.label[c];
        const int rows = block_rows(lab, N);
        double *fo = A.f + row0;
        double *so = SCALE ? A.fscale + row0 : nullptr;
        if (F.por[c] < kPorTiny) {
            for (int r = 0; r < rows; r++) {
                fo[r] = 0;
                if (so) so[r] = 0;
            }
            continue;
        }
        const int ix = (int)(c % s.nx), iy = (int)((c / s.nx) % s.ny), iz = (int)(c / ((long)s.nx * s.ny));
        const double di = geo.di[ix], dj = geo.dj[iy], dk = geo.dk[iz];
        const double Vb = di * dj * dk;
        const double porpor = porpor_at(F, s, c);
        const double Mpor = porpor_at(M, s, c), Fpor = porpor_at(Fr, s, c);
        const double tor = A.tor[c];
        // ---- two-phase fugacity rows
        int r = 0;
        if (lab == 0) {
            const double Po = F.P[n + c], Pg = F.P[2 * n + c];
            const PhaseFug<N> fl(A.a.g, F.x, n, c, Po, F.rho[c]);
            const PhaseFug<N> fg(A.a.g, F.y, n, c, Pg, F.rho[n + c]);
#pragma unroll
            for (int i = 0; i < N; i++) {
                const double phiL = fl.coeff(A.a.g.f, i);
                const double phiG = fg.coeff(A.a.g.f, i);
                const double a1 = F.x[(long)i * n + c] * Po * phiL, a2 = F.y[(long)i * n + c] * Pg * phiG;
                fo[r] = a1 - a2;
                if (so) so[r] = fabs(a1) + fabs(a2);
                r++;
            }
        }
        // ---- faces: advective factors per phase (oil 0, gas 1)
        Face fc[6];
        const int nf = cell_faces<N>(A, c, ix, iy, iz, fc);
        unsigned bits = 0;
        // the water row's face terms, summed in face order as the row adds them
        double RW = 0, SW = 0;
        for (int q = 0; q < nf; q++) {
            const Face &e = fc[q];
            sf.nb[q][t] = (int)e.nb;
            if (e.sgn > 0) bits |= 1u << q;
            const long plane = (long)e.d * n + e.tc;
            const double dH = e.sgn > 0 ? geo.blockH[e.nb] - geo.blockH[c] : geo.blockH[c] - geo.blockH[e.nb];
            for (int p = 0; p < 2; p++) {
                const double Tp = F.trans[(long)(p * 3) * n + plane];
                const double Tg = F.trans[(long)((2 + p) * 3) * n + plane];
                const double Pc_ = F.P[(1 + p) * n + c], Pn_ = F.P[(1 + p) * n + e.nb];
                const int tS = F.transS[(long)(p * 3) * n + plane];
                const int pq = p * 6 + q;
                if (e.sgn > 0) {
                    sf.kp[pq][t] = Tp * (Pn_ - Pc_);
                    sf.kg[pq][t] = Tg * dH;
                    sf.up[pq][t] = (int)(tS ? e.nb : c);
                } else {
                    sf.kp[pq][t] = -(Tp * (Pc_ - Pn_));
                    sf.kg[pq][t] = -(Tg * dH);
                    sf.up[pq][t] = (int)(tS ? c : e.nb);
                }
            }
            const double Tw = F.wtran[plane];
            const double dPw = e.sgn > 0 ? F.P[e.nb] - F.P[c] : F.P[c] - F.P[e.nb];
            const double kw = e.sgn * (Tw * dPw + kGAcc * s.wat_ro * Tw * dH);
            RW += kw;
            SW += fabs(kw);
        }
        // ---- matrix-fracture advective transfer (identical value, opposite sign)
        const double sgnT = med == 0 ? 1.0 : -1.0;
        const double SF2 = 4 * A.k.sigma * (M.perm[c] / (di * di) + M.perm[n + c] / (dj * dj) + M.perm[2 * n + c] / (dk * dk));
        const double SF1 = A.k.diff_off ? 0.0 : 4 * A.k.sigma * ((1 / (di * di)) + (1 / (dj * dj)) + (1 / (dk * dk)));
        const double SF3 = A.k.diff_off ? 0.0 : 4 * A.k.sigma * ((1 / di) + (1 / dj) + (1 / dk)) / A.k.lf;
        const double kr_o = M.P[n + c] >= Fr.P[n + c] ? M.kr[n + c] : Fr.kr[n + c];
        const double kr_g = M.P[2 * n + c] >= Fr.P[2 * n + c] ? M.kr[2 * n + c] : Fr.kr[2 * n + c];
        const double kr_w = M.P[c] >= Fr.P[c] ? M.kr[c] : Fr.kr[c];
        const double mubar_o = (M.mu[c] * Mpor + Fr.mu[c] * Fpor) / (Mpor + Fpor);
        const double mubar_g = (M.mu[n + c] * Mpor + Fr.mu[n + c] * Fpor) / (Mpor + Fpor);
        const double conv_o = kSIC * M.rho[c] * SF2 * Vb * kr_o / mubar_o * (Fr.P[n + c] - M.P[n + c]);
        const double conv_g = kSIC * M.rho[n + c] * SF2 * Vb * kr_g / mubar_g *
                              ((Fr.P[2 * n + c] - M.P[2 * n + c]) + (Fr.pc[n + c] - M.pc[n + c]));
        const double conv_w = kSIC * wfac * SF2 * kr_w / s.wat_mu * Vb * ((Fr.P[c] - M.P[c]) + (M.pc[c] - Fr.pc[c]));
        // ---- wells
        WellRates wr;
        well_rates<N>(A, med, c, ix, iy, iz, wr);
        // ---- diffusive transfer coefficients of this continuum's rows
        const signed char lm = M.label[c], lf = Fr.label[c];
        // matrix diffusion factors (SF1 terms) and fracture factors (SF3 terms)
        const double dmo = SF1 * Vb * Mpor / tor * M.sat[n + c] * M.rho[c];
        const double dmg = SF1 * Vb * Mpor / tor * M.sat[2 * n + c] * M.rho[n + c];
        const double dfo = SF3 * Vb * Fpor / tor * Fr.sat[n + c] * Fr.rho[c];
        const double dfg = SF3 * Vb * Fpor / tor * Fr.sat[2 * n + c] * Fr.rho[n + c];
        const double dCoefl = lab == -1 ? 0.0 : 1.0, dCoefg = lab == 1 ? 0.0 : 1.0;
        // ---- intra-continuum diffusion: the factor of each (face, phase)
        // that does not depend on the component, AAd / BBd * NNd of the
        // reference's DTran = AAd / BBd * NNd * Dup (formed once here, applied
        // per component row below with the same evaluation order)
        for (int q = 0; q < nf; q++) {
            const Face &e = fc[q];
            const long nb = e.nb;
            const double porpor2 = porpor_at(F, s, nb);
            const double NNd = e.area2 / (e.dn + e.dl);
            const signed char lnb = F.label[nb];
            if (F.por[c] < kPorTiny || F.por[nb] < kPorTiny) bits |= 1u << (6 + q);
            for (int p = 0; p < 2; p++) {
                const double Coef = p ? (lnb == 1 ? 0.0 : 1.0) : (lnb == -1 ? 0.0 : 1.0);
                const double dC = p ? dCoefg : dCoefl;
                double AAd = F.rho[p * n + nb] * e.dn * Coef + F.rho[p * n + c] * e.dl * dC;
                AAd *= (F.sat[(1 + p) * n + nb] * e.dn * Coef + F.sat[(1 + p) * n + c] * e.dl * dC) / (e.dn + e.dl);
                const double tn = med == 0 ? A.tor[nb] : 1.0, tc_ = med == 0 ? tor : 1.0;
                const double BBd = tn * e.dn * Coef / porpor2 + tc_ * e.dl * dC / porpor;
                sf.db[p * 6 + q][t] = AAd / BBd * NNd;
                if (Coef == 0 && dC == 0) bits |= 1u << (12 + p * 6 + q);
            }
        }
        // ---- component balances (first N-1 components)
        for (int i = 0; i < N - 1; i++, r++) {
            double R = 0, sc = 0;
            auto add = [&](double v) {
                R += v;
                if (SCALE) sc += fabs(v);
            };
            for (int p = 0; p < 2; p++) {
                const double *w = p ? F.y : F.x;
                for (int q = 0; q < nf; q++) add(w[(long)i * n + sf.up[p * 6 + q][t]] * sf.kp[p * 6 + q][t]);
            }
            for (int p = 0; p < 2; p++) {
                const double *w = p ? F.y : F.x;
                for (int q = 0; q < nf; q++) add(w[(long)i * n + sf.up[p * 6 + q][t]] * sf.kg[p * 6 + q][t]);
            }
            add(sgnT * M.x[(long)i * n + c] * conv_o);
            add(sgnT * M.y[(long)i * n + c] * conv_g);
            const double xm = M.x[(long)i * n + c], ym = M.y[(long)i * n + c];
            const double xf = Fr.x[(long)i * n + c], yf = Fr.y[(long)i * n + c];
            const double Dmo = M.diff[(long)(2 * i) * n + c], Dmg = M.diff[(long)(2 * i + 1) * n + c];
            const double Dfo = Fr.diff[(long)(2 * i) * n + c], Dfg = Fr.diff[(long)(2 * i + 1) * n + c];
            if (med == 0) {
                // EdgeComp is identically zero (the reference overwrites it)
                const double mo = dmo * Dmo, mg = dmg * Dmg;
                if (lm == 1 && lf == 1) add(mo * (xf - xm));
                if (lm == -1 && lf == -1) add(mg * (yf - ym));
                if (lm == 0 && lf == 0) { add(mo * (xf - xm)); add(mg * (yf - ym)); }
                if (lm == 1 && lf == -1) add(mo * (0 - xm));
                if (lm == -1 && lf == 1) add(mg * (0 - ym));
                if (lm == 0 && lf == 1) { add(mg * (0 - ym)); add(mo * (xf - xm)); }
                if (lm == 0 && lf == -1) { add(mg * (yf - ym)); add(mo * (0 - xm)); }
                if (lm == 1 && lf == 0) { add(mo * (0 - xm)); add(mo * (xf - xm)); }
                if (lm == -1 && lf == 0) { add(mg * (yf - ym)); add(mg * (0 - ym)); }
            } else {
                const double mo = dmo * Dmo, mg = dmg * Dmg, fo_ = dfo * Dfo, fg = dfg * Dfg;
                if (lm == 1 && lf == 1) add(-(mo * (xf - xm)));
                if (lm == -1 && lf == -1) add(-(mg * (yf - ym)));
                if (lm == 0 && lf == 0) { add(-(mo * (xf - xm))); add(-(mg * (yf - ym))); }
                if (lm == 1 && lf == -1) add(-(fg * (yf - 0)));
                if (lm == -1 && lf == 1) add(-(fo_ * (xf - 0)));
                if (lm == 0 && lf == 1) { add(-(fo_ * (xf - 0))); add(-(mo * (xf - xm))); }
                if (lm == 0 && lf == -1) { add(-(mg * (yf - ym))); add(-(fg * (yf - 0))); }
                if (lm == 1 && lf == 0) { add(-(fg * (yf - 0))); add(-(mo * (xf - xm))); }
                if (lm == -1 && lf == 0) { add(-(mg * (yf - ym))); add(-(fo_ * (xf - 0))); }
            }
            // wells
            double oComp = F.x[(long)i * n + c], gComp = F.y[(long)i * n + c];
            if (wr.iwell >= 0) {
                oComp = A.w.ws[wr.iwell].xo[i];
                gComp = A.w.ws[wr.iwell].yg[i];
            }
            add(oComp * wr.Qo + gComp * wr.Qg);
            // intra-continuum diffusion
            for (int q = 0; q < nf; q++) {
                const long nb = sf.nb[q][t];
                for (int p = 0; p < 2; p++) {
                    const double *w = p ? F.y : F.x;
                    const double wn = w[(long)i * n + nb], wc = w[(long)i * n + c];
                    double Dup = wn > wc ? F.diff[(long)(2 * i + p) * n + nb] : F.diff[(long)(2 * i + p) * n + c];
                    if (bits & (1u << (6 + q))) Dup = 0;
                    double DTran = sf.db[p * 6 + q][t] * Dup;
                    if (bits & (1u << (12 + p * 6 + q))) DTran = 0;
                    add((bits & (1u << q)) ? DTran * (wn - wc) : -(DTran * (wc - wn)));
                }
            }
            fo[r] = 0 - R;   // LSide: the accumulation at the linearisation point minus itself
            if (SCALE) so[r] = sc;
        }
        // ---- total hydrocarbon
        {
            double R = 0, sc = 0;
            auto add = [&](double v) {
                R += v;
                sc += fabs(v);
            };
            for (int p = 0; p < 2; p++)
                for (int q = 0; q < nf; q++) add(sf.kp[p * 6 + q][t]);
            for (int p = 0; p < 2; p++)
                for (int q = 0; q < nf; q++) add(sf.kg[p * 6 + q][t]);
            add(sgnT * conv_o);
            add(sgnT * conv_g);
            add(wr.Qo + wr.Qg);
            fo[r] = 0 - R;
            if (so) so[r] = sc;
            r++;
        }
        // ---- water
        {
            double R = RW, sc = SW;
            R += sgnT * conv_w;
            sc += fabs(conv_w);
            R += wr.Qw;
            sc += fabs(wr.Qw);
            fo[r] = 0 - R;
            if (so) so[r] = sc;
            r++;
        }
        // ---- constraints
        auto sum_w = [&](const double *w) {
            double t = 0;
            for (int i = 0; i < N; i++) t += w[(long)i * n + c];
            return t;
        };
        if (lab == 0) {
            fo[r] = sum_w(F.x) - 1;
            if (so) so[r] = 1;
            r++;
            fo[r] = sum_w(F.y) - 1;
            if (so) so[r] = 1;
            r++;
        } else {
            fo[r] = sum_w(lab == 1 ? F.x : F.y) - 1;
            if (so) so[r] = 1;
            r++;
        }
        fo[r] = F.sat[c] + F.sat[n + c] + F.sat[2 * n + c] - 1;
        if (so) so[r] = 1;
    }
}

// ---------------------------------------------------------------------------
// Vector-Jacobian product of the residual with the matrix continuum's
// per-cell log-permeability theta_c = ln k_c (k_x, k_y, k_z of matrix cell c
// scaled together): gk[c] = sum_rows lambda_r dF_r/d theta_c at the current
// state.  The reference has no adjoint; this differentiates its residual
// (IteratorFunction, compsim/Petsc_Functions.cpp:10-6895) through the two
// places the matrix permeability enters it:
//  * the interface transmissibility of each matrix face, harmonic in the two
//    cells' permeabilities (IFK_Calc, compsim/Init_Calcs.cpp:21-46), which
//    multiplies every advective face term (Calc_Transes,
//    compsim/Do_Cycle.cpp:800-1416): d ln T_f/d theta_a =
//    (h_a/k_a)/(h_a/k_a + h_b/k_b);
//  * the convective matrix-fracture shape factor 4 sigma sum_d k_d/L_d^2
//    (compsim/Init_Calcs.cpp:970-983), linear in the cell's permeability.
// The face terms are those residual_kernel forms for the matrix rows; a face
// enters its two cells' rows with opposite signs, so a thread evaluates each
// of its faces once and weights both cells' multipliers (no atomics; the
// result is deterministic).  Well productivity indices (Peaceman, through
// sqrt(k_x k_y)) are held fixed: this product is for the grid's flux and
// transfer terms.
template <int N>
__global__ void __launch_bounds__(128) residual_logk_vjp_kernel(const __grid_constant__ AsmArgs<N> A,
                                                                const double *lam, double *gk) {
    const GridScalars &s = A.a.s;
    const GridGeom &geo = A.a.geo;
    const long n = s.cells;
    const double wfac = s.wat_ro * kWatMRo;
    const MediumFields &M = A.a.m[0], &Fr = A.a.m[1];
    // lambda of block b's i-th component row, total row (i = N-1), water row (i = N)
    auto lam_row = [&](long b, int i) -> double {
        const signed char lb = b >= n ? Fr.label[b - n] : M.label[b];
        return lam[A.rowoff[b] + (lb == 0 ? N : 0) + i];
    };
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
        const int ix = (int)(c % s.nx), iy = (int)((c / s.nx) % s.ny), iz = (int)(c / ((long)s.nx * s.ny));
        const bool act_c = M.por[c] >= kPorTiny;
        double g = 0;
        Face fc[6];
        const int nf = cell_faces<N>(A, c, ix, iy, iz, fc);
        for (int q = 0; q < nf; q++) {
            const Face &e = fc[q];
            const bool act_nb = M.por[e.nb] >= kPorTiny;
            if (!act_c && !act_nb) continue;
            const long plane = (long)e.d * n + e.tc;
            const double dH = e.sgn > 0 ? geo.blockH[e.nb] - geo.blockH[c] : geo.blockH[c] - geo.blockH[e.nb];
            double KPG[2];
            long up[2];
            for (int p = 0; p < 2; p++) {
                const double Tp = M.trans[(long)(p * 3) * n + plane];
                const double Tg = M.trans[(long)((2 + p) * 3) * n + plane];
                const double Pc_ = M.P[(1 + p) * n + c], Pn_ = M.P[(1 + p) * n + e.nb];
                const int tS = M.transS[(long)(p * 3) * n + plane];
                if (e.sgn > 0) {
                    KPG[p] = Tp * (Pn_ - Pc_) + Tg * dH;
                    up[p] = tS ? e.nb : c;
                } else {
                    KPG[p] = -(Tp * (Pc_ - Pn_)) - Tg * dH;
                    up[p] = tS ? c : e.nb;
                }
            }
            const double Tw = M.wtran[plane];
            const double dPw = e.sgn > 0 ? M.P[e.nb] - M.P[c] : M.P[c] - M.P[e.nb];
            const double KW = e.sgn * (Tw * dPw + kGAcc * s.wat_ro * Tw * dH);
            // this face's terms in c's rows; the neighbour's rows hold the negatives
            double S = 0;
            for (int i = 0; i < N - 1; i++) {
                const double term = M.x[(long)i * n + up[0]] * KPG[0] + M.y[(long)i * n + up[1]] * KPG[1];
                S += ((act_c ? lam_row(c, i) : 0.0) - (act_nb ? lam_row(e.nb, i) : 0.0)) * term;
            }
            S += ((act_c ? lam_row(c, N - 1) : 0.0) - (act_nb ? lam_row(e.nb, N - 1) : 0.0)) * (KPG[0] + KPG[1]);
            S += ((act_c ? lam_row(c, N) : 0.0) - (act_nb ? lam_row(e.nb, N) : 0.0)) * KW;
            const double hc = e.dl / M.perm[(long)e.d * n + c], hn = e.dn / M.perm[(long)e.d * n + e.nb];
            g += hc / (hc + hn) * S;
        }
        // matrix-fracture convective transfer: +conv in the matrix rows, -conv in the fracture rows
        const bool act_f = Fr.por[c] >= kPorTiny;
        if (act_c || act_f) {
            const double di = geo.di[ix], dj = geo.dj[iy], dk = geo.dk[iz];
            const double Vb = di * dj * dk;
            const double Mpor = porpor_at(M, s, c), Fpor = porpor_at(Fr, s, c);
            const double SF2 = 4 * A.k.sigma *
                               (M.perm[c] / (di * di) + M.perm[n + c] / (dj * dj) + M.perm[2 * n + c] / (dk * dk));
            const double kr_o = M.P[n + c] >= Fr.P[n + c] ? M.kr[n + c] : Fr.kr[n + c];
            const double kr_g = M.P[2 * n + c] >= Fr.P[2 * n + c] ? M.kr[2 * n + c] : Fr.kr[2 * n + c];
            const double kr_w = M.P[c] >= Fr.P[c] ? M.kr[c] : Fr.kr[c];
            const double mubar_o = (M.mu[c] * Mpor + Fr.mu[c] * Fpor) / (Mpor + Fpor);
            const double mubar_g = (M.mu[n + c] * Mpor + Fr.mu[n + c] * Fpor) / (Mpor + Fpor);
            const double conv_o = kSIC * M.rho[c] * SF2 * Vb * kr_o / mubar_o * (Fr.P[n + c] - M.P[n + c]);
            const double conv_g = kSIC * M.rho[n + c] * SF2 * Vb * kr_g / mubar_g *
                                  ((Fr.P[2 * n + c] - M.P[2 * n + c]) + (Fr.pc[n + c] - M.pc[n + c]));
            const double conv_w =
                kSIC * wfac * SF2 * kr_w / s.wat_mu * Vb * ((Fr.P[c] - M.P[c]) + (M.pc[c] - Fr.pc[c]));
            double S = 0;
            for (int i = 0; i < N - 1; i++) {
                const double term = M.x[(long)i * n + c] * conv_o + M.y[(long)i * n + c] * conv_g;
                S += ((act_c ? lam_row(c, i) : 0.0) - (act_f ? lam_row(n + c, i) : 0.0)) * term;
            }
            S += ((act_c ? lam_row(c, N - 1) : 0.0) - (act_f ? lam_row(n + c, N - 1) : 0.0)) * (conv_o + conv_g);
            S += ((act_c ? lam_row(c, N) : 0.0) - (act_f ? lam_row(n + c, N) : 0.0)) * conv_w;
            g += S;
        }
        gk[c] = -g;   // the residual is F = LSide - RSide with the flux terms in RSide
    }
}

}  // namespace osr
