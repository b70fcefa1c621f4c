// Successive-substitution flash with an inner Rachford-Rice Newton, and the
// fugacity-derivative pass, as FP64 CUDA kernels for sm_100a.
//
// Algorithm: the reference's SuccFalsh (compsim/Init_Calcs.cpp:571-738):
//   K_i = Pc_i/P exp(5.37 (1 + w_i)(1 - Tc_i/T))                (Wilson)
//   repeat (at most 500 times, until |L_k - L_{k-1}| <= 1e-14):
//     L = 0.6; Newton on sum_i z_i (1-K_i)/(L + (1-L) K_i) = 0
//       (at most 100 steps, until step^2 <= 1e-8); clamp L to [0,1]
//     x_i = z_i/(L + K_i (1-L)), y_i = K_i x_i    (K_i < 0 flags a component
//       the vapour cannot hold: x_i = 0, y_i = z_i/(1-L))
//     Z_l, Z_v from the cubic; K_i *= x_i phi_i^L / (y_i phi_i^V)
//   label = -1 (vapour only) if |L| < 1e-20, +1 (liquid only) if |1-L| < 1e-20,
//   else 0 (two-phase).
//
// Work distribution.  Per-cell cost is heavy-tailed (most single-phase cells
// need 2-3 substitution steps, two-phase cells tens to hundreds, and each step
// runs 1 to 100 Newton steps), so a thread-per-cell grid would idle most lanes
// of a warp behind its slowest cell.  The batched kernel is persistent: every
// lane runs a small state machine (fetch cell -> Newton steps -> substitution
// step -> ...), claims a new cell from a global work counter as soon as its
// cell converges, and the warp runs the expensive substitution step only when
// enough lanes are ready for it, so that step executes with most lanes busy.
// The plain kernel (one thread per cell, no queue) is kept as the baseline the
// batched form is measured against.
#pragma once

// Resident 128-thread CTAs per SM the queue kernel is compiled for (bounds
// its registers).
#ifndef OSR_FLASH_MIN_BLOCKS
#define OSR_FLASH_MIN_BLOCKS 3
#endif
#include "eos_device.cuh"

namespace osr {

// Device pointers of one flash batch.  Per-component fields are [nc][n].
struct FlashIO {
    const double *P, *T, *z;
    long n;
    signed char *label;
    double *L, *x, *y, *Zl, *Zg;
    int *iters, *rr_iters;  // optional (may be null)
};

template <int N>
struct FlashArgs {
    FluidTable<N> f;
    FlashIO io;
};

// Bound beyond which a Rachford-Rice Newton run provably ends outside [0,1].
// Every term of F(L) = sum_i z_i (1-K_i)/(L + (1-L) K_i) is z_i/(L + c_i) with
// c_i = K_i/(1-K_i) (c_i = -1 for a flagged K_i < 0; K_i = 1 contributes 0).
// For |L| > 2 max|c_i| + 2 every denominator has the sign of L, so the Newton
// step L - F/F' = L + (weighted mean of L + c_i) moves L further out by more
// than 1e-4 each time: the loop runs to its 100-step cap and the clamp that
// follows (compsim/Init_Calcs.cpp:608-615) gives 1 for L > 0 and 0 for L < 0
// whatever the remaining steps do.  Stopping there returns the same clamped L.
template <int N>
__device__ __forceinline__ double rr_bound(const double *K) {
    double M = 1;
#pragma unroll
    for (int i = 0; i < N; i++)
        if (K[i] >= 0 && K[i] != 1) M = fmax(M, fabs(K[i] / (1 - K[i])));
    return 2 * M + 2;
}

// One Rachford-Rice Newton step (compsim/Init_Calcs.cpp:595-605), one
// division per component, the sums as a pairwise tree.  Returns the step t;
// L is updated in place.
template <int N, bool Fast>
__device__ __forceinline__ double rr_step_impl(const double *K, const double *z, double &L, bool &ok) {
    double zt[N], zq[N];
    const double omL = 1 - L;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const bool pos = K[i] >= 0;
        double num = pos ? 1 - K[i] : 1.0;
        double den = pos ? L + omL * K[i] : L - 1;
        double td;
        if (Fast) {
            ok &= qdiv_ok(num, den);
            td = qdiv(num, den);
        } else {
            td = num / den;
        }
        zt[i] = z[i] * td;
        zq[i] = zt[i] * td;
    }
#pragma unroll
    for (int w = 1; w < N; w *= 2)
#pragma unroll
        for (int i = 0; i + w < N; i += 2 * w) {
            zt[i] += zt[i + w];
            zq[i] += zq[i + w];
        }
    double F = zt[0], dF = -zq[0];
    double t;
    if (Fast) {
        ok &= qdiv_ok(F, dF);
        t = qdiv(F, dF);
    } else {
        t = F / dF;
    }
    return t;
}

template <int N>
__device__ __forceinline__ double rr_step(const double *K, const double *z, double &L) {
    bool ok = true;
    double t = rr_step_impl<N, true>(K, z, L, ok);
    if (!ok) t = rr_step_impl<N, false>(K, z, L, ok);
    L -= t;
    return t;
}

// The whole Newton run of one substitution step; returns the step count the
// reference would take (the provably divergent tail is cut, see rr_bound).
template <int N>
__device__ __forceinline__ int rr_solve(const double *K, const double *z, double &L) {
    const double big = rr_bound<N>(K);
    L = 0.6;
    int j = 0;
    double t;
    do {
        t = rr_step<N>(K, z, L);
        j++;
        if (fabs(L) > big) return kRRMaxIt;
    } while ((t * t > kRRTol) && (j < kRRMaxIt));
    return j;
}

// One substitution step after the Newton loop: clamp L, form x, y, solve both
// cubics and update K (compsim/Init_Calcs.cpp:608-712).  Returns |Lb - L|.
// The Fast instantiation uses the branch-free quotients and reports through
// ok whether every operand was in range; K is written only by the caller.
template <int N, bool Fast>
__device__ __forceinline__ double ss_update_impl(const FluidTable<N> &f, const double *sa, double P, double T,
                                                 const double *z, const double *K, double *Kn, double L0,
                                                 double &L, double Lb, double *x, double *y, double &Zl,
                                                 double &Zg, bool &ok) {
    auto DIV = [&](double a, double b) -> double {
        if (Fast) {
            ok &= qdiv_ok(a, b);
            return qdiv(a, b);
        }
        return a / b;
    };
    L = L0;
    if (L > 1) L = 1;
    else if (L < 0) L = 0;
    double es = fabs(Lb - L);
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (K[i] >= 0) {
            x[i] = DIV(z[i], L + K[i] * (1 - L));
            y[i] = K[i] * x[i];
        } else {
            x[i] = 0;
            y[i] = DIV(z[i], 1 - L);
        }
    }
    // Mixing rule: with u_i = w_i sqrt(a_i) and v_i = sum_j (1-k_ij) u_j,
    // sum_i sum_j w_i w_j sqrt(a_i a_j)(1-k_ij) = sum_i u_i v_i and the
    // per-component sums sum_j w_j sqrt(a_i a_j)(1-k_ij) = sqrt(a_i) v_i.
    double ul[N], ug[N], vl[N], vg[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        ul[i] = x[i] * sa[i];
        ug[i] = y[i] * sa[i];
    }
    double Cal = 0, Cag = 0, Cbl = 0, Cbg = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        double sl = 0, sg = 0;
#pragma unroll
        for (int j = 0; j < N; j++) {
            sl += f.bic[i * N + j] * ul[j];
            sg += f.bic[i * N + j] * ug[j];
        }
        vl[i] = sl;
        vg[i] = sg;
        Cal += ul[i] * sl;
        Cag += ug[i] * sg;
        Cbl += x[i] * f.b[i];
        Cbg += y[i] * f.b[i];
    }
    const double pa = P / (kR * kR * T * T), pb = P / (kR * T);
    double Al = Cal * pa, Bl = Cbl * pb, Ag = Cag * pa, Bg = Cbg * pb;
    const bool srk = f.srk != 0;
    Zl = phase_z(Al, Bl, srk, false);
    Zg = phase_z(Ag, Bg, srk, true);
    const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
    // i-independent parts of ln(phi_i) (the reference re-evaluates them per i)
    double DDl = DIV(Al, Bl * (d1 - d2)), DDg = DIV(Ag, Bg * (d1 - d2));
    double FFl = log(DIV(Zl + d2 * Bl, Zl + d1 * Bl)), FFg = log(DIV(Zg + d2 * Bg, Zg + d1 * Bg));
    double cl = log(Zl - Bl), cg = log(Zg - Bg);
    double rCal = DIV(2.0, Cal), rCag = DIV(2.0, Cag), rCbl = DIV(1.0, Cbl), rCbg = DIV(1.0, Cbg);
    double DFl = DDl * FFl, DFg = DDg * FFg;
    double lnl[N], lng[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        double t1l = f.b[i] * rCbl, t1g = f.b[i] * rCbg;
        double EEl = sa[i] * vl[i] * rCal - t1l;
        double EEg = sa[i] * vg[i] * rCag - t1g;
        lnl[i] = t1l * (Zl - 1) - cl + DFl * EEl;
        lng[i] = t1g * (Zg - 1) - cg + DFg * EEg;
    }
    // K_i x_i phi_i^L / (y_i phi_i^V) with y_i = K_i x_i is phi_i^L / phi_i^V:
    // one exponential per component, evaluated for all components without
    // branching; components with a zero, infinite or extreme factor take the
    // reference's own form (and its zero/NaN rules) in one separate pass.
    bool plain = true;
#pragma unroll
    for (int i = 0; i < N; i++) {
        double d = lnl[i] - lng[i];
        bool fast = K[i] > 0 && x[i] > 0 && y[i] > 0 && x[i] < 1e300 && y[i] < 1e300 && fabs(lnl[i]) < 700 &&
                    fabs(lng[i]) < 700 && fabs(d) < 700;
        plain &= fast || z[i] == 0;
        double e = exp(fast ? d : 0.0);
        Kn[i] = (z[i] != 0 && fast) ? e : K[i];
    }
    if (!plain) {
#pragma unroll
        for (int i = 0; i < N; i++) {
            double d = lnl[i] - lng[i];
            bool fast = K[i] > 0 && x[i] > 0 && y[i] > 0 && x[i] < 1e300 && y[i] < 1e300 &&
                        fabs(lnl[i]) < 700 && fabs(lng[i]) < 700 && fabs(d) < 700;
            if (z[i] != 0 && !fast) {
                double fL = x[i] * exp(lnl[i]), fG = y[i] * exp(lng[i]);
                if (fG != 0) Kn[i] = K[i] * (fL / fG);
                else Kn[i] = -1;
                if (fL != fL) Kn[i] = -1;
                if (fG != fG) Kn[i] = 1;
            }
        }
    }
    return es;
}

template <int N>
__device__ __forceinline__ double ss_update(const FluidTable<N> &f, const double *sa, double P, double T,
                                            const double *z, double *K, double &L, double &Lb, double *x,
                                            double *y, double &Zl, double &Zg) {
    bool ok = true;
    double Kn[N];
    const double L0 = L;
    double es = ss_update_impl<N, true>(f, sa, P, T, z, K, Kn, L0, L, Lb, x, y, Zl, Zg, ok);
    if (!ok) es = ss_update_impl<N, false>(f, sa, P, T, z, K, Kn, L0, L, Lb, x, y, Zl, Zg, ok);
#pragma unroll
    for (int i = 0; i < N; i++) K[i] = Kn[i];
    Lb = L;
    return es;
}

template <int N>
__device__ __forceinline__ void flash_init(const FluidTable<N> &f, double P, double T, double *K, double *sa) {
#pragma unroll
    for (int i = 0; i < N; i++) K[i] = (f.pc[i] / P) * exp(f.wil[i] * (1 - f.tc[i] / T));
    sqrt_a<N>(f, T, sa);
}

__device__ __forceinline__ signed char flash_label(double L) {
    if (fabs(L) < kLZero) return -1;
    if (fabs(1 - L) < kLZero) return 1;
    return 0;
}

template <int N>
__device__ __forceinline__ void flash_store(const FlashIO &io, long c, double L, const double *x, const double *y,
                                            double Zl, double Zg, int k, int rr) {
    io.label[c] = flash_label(L);
    io.L[c] = L;
#pragma unroll
    for (int i = 0; i < N; i++) {
        io.x[(long)i * io.n + c] = x[i];
        io.y[(long)i * io.n + c] = y[i];
    }
    io.Zl[c] = Zl;
    io.Zg[c] = Zg;
    if (io.iters) io.iters[c] = k;
    if (io.rr_iters) io.rr_iters[c] = rr;
}

// Plain form: one thread per cell, the whole iteration in one thread.
template <int N>
__global__ void __launch_bounds__(128) flash_plain_kernel(const __grid_constant__ FlashArgs<N> a) {
    long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.io.n) return;
    const FlashIO &io = a.io;
    double P = io.P[c], T = io.T[c];
    double z[N], K[N], sa[N], x[N], y[N];
#pragma unroll
    for (int i = 0; i < N; i++) z[i] = io.z[(long)i * io.n + c];
    flash_init<N>(a.f, P, T, K, sa);
    double L = 0, Lb = 10, Zl = 0, Zg = 0, es;
    int k = 0, rr = 0;
    do {
        rr += rr_solve<N>(K, z, L);
        es = ss_update<N>(a.f, sa, P, T, z, K, L, Lb, x, y, Zl, Zg);
        k++;
    } while ((es > kSSTol) && (k < kSSMaxIt));
    flash_store<N>(io, c, L, x, y, Zl, Zg, k, rr);
}

enum : int { kFetch = 0, kNewton = 1, kReady = 2, kDone = 3 };

// A list of cells in flight: their substitution state, so that a later pass
// resumes each exactly where it stopped (K, iteration counts, previous L).
struct ParkList {
    long *cell;          // [cap] cell index
    int *k, *rr;         // [cap] SS steps so far, Newton steps so far
    double *Lb;          // [cap] L of the last substitution step
    double *K;           // [nc][cap] K-values
    long cap;
};

template <int N>
struct QueueArgs {
    FluidTable<N> f;
    FlashIO io;
    ParkList src, dst;           // resume from src (pass > 0); park into dst
    const unsigned *src_count;   // cells in src (pass > 0)
    unsigned *dst_count;         // cells parked into dst
    unsigned long long *head;    // work-queue head of this pass; zero at launch
    int ss_batch;                // ready lanes needed before a substitution step runs ...
    int max_wait;                // ... or Newton trips the ready lanes have waited
    int park_at;                 // park a cell still running once it reaches this many SS steps
    int first;                   // 1: take cells [0, n) fresh; 0: resume src
    // several instances (fluids) of one component count: cells
    // [inst_start[i], inst_start[i+1]) use tables[i]
    const FluidTable<N> *tables;
    const long *inst_start;
    int n_inst;
};

// Instance of cell c: the largest i with start[i] <= c.
__device__ __forceinline__ int find_instance(const long *start, int n_inst, long c) {
    int lo = 0, hi = n_inst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The component table of a cell: the kernel parameter, or its instance's.
template <int N, bool MULTI, class Args>
__device__ __forceinline__ const FluidTable<N> &table_of(const Args &a, int inst) {
    if constexpr (MULTI) return a.tables[inst];
    else return a.f;
}

// Batched form: persistent warps, a per-lane state machine and a global work
// queue, run as a sequence of passes.  The first pass takes every cell; a
// cell still running when it reaches park_at substitution steps is parked
// (its state written to dst) and its lane takes the next cell.  Each later
// pass resumes the parked cells of the previous one with a doubled limit, so
// every pass starts with fully populated warps instead of draining a few
// long cells through mostly idle warps.
template <int N, bool MULTI>
__device__ __forceinline__ void queue_pass(const QueueArgs<N> &a) {
    constexpr unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const FlashIO &io = a.io;
    const long total = a.first ? io.n : (long)__ldcg(a.src_count);
    int mode = kFetch;
    long c = -1;
    double P = 0, T = 0, L = 0, Lb = 10;
    double z[N], K[N], sa[N];
    int j = 0, k = 0, rr = 0;
    int waited = 0;  // warp-uniform: Newton trips since ready lanes appeared
    int inst = 0;
    double big = 0;
#pragma unroll
    for (int i = 0; i < N; i++) z[i] = K[i] = sa[i] = 0;
    for (;;) {
        unsigned need = __ballot_sync(kFull, mode == kFetch);
        if (need) {
            int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(a.head, (unsigned long long)__popc(need));
            base = __shfl_sync(kFull, base, leader);
            if (mode == kFetch) {
                long q = (long)base + __popc(need & ((1u << lane) - 1));
                if (q < total) {
                    if (a.first) {
                        c = q;
                        k = 0;
                        rr = 0;
                        Lb = 10;
                    } else {
                        c = __ldcg(a.src.cell + q);
                        k = __ldcg(a.src.k + q);
                        rr = __ldcg(a.src.rr + q);
                        Lb = __ldcg(a.src.Lb + q);
#pragma unroll
                        for (int i = 0; i < N; i++) K[i] = __ldcg(a.src.K + (long)i * a.src.cap + q);
                    }
                    P = io.P[c];
                    T = io.T[c];
#pragma unroll
                    for (int i = 0; i < N; i++) z[i] = io.z[(long)i * io.n + c];
                    if constexpr (MULTI) inst = find_instance(a.inst_start, a.n_inst, c);
                    if (a.first) flash_init<N>(table_of<N, MULTI>(a, inst), P, T, K, sa);
                    else sqrt_a<N>(table_of<N, MULTI>(a, inst), T, sa);
                    L = 0.6;
                    j = 0;
                    big = rr_bound<N>(K);
                    mode = kNewton;
                } else {
                    mode = kDone;
                }
            }
        }
        if (__ballot_sync(kFull, mode != kDone) == 0) break;
        if (mode == kNewton) {
            double t = rr_step<N>(K, z, L);
            j++;
            if (fabs(L) > big) {
                j = kRRMaxIt;  // provably divergent: the reference runs to its cap
                mode = kReady;
            } else if (!((t * t > kRRTol) && (j < kRRMaxIt))) {
                mode = kReady;
            }
        }
        unsigned ready = __ballot_sync(kFull, mode == kReady);
        unsigned newton = __ballot_sync(kFull, mode == kNewton);
        if (ready != 0) waited++;
        if (ready != 0 && (__popc(ready) >= a.ss_batch || newton == 0 || waited > a.max_wait)) {
            waited = 0;
            if (mode == kReady) {
                double x[N], y[N], Zl, Zg;
                double es = ss_update<N>(table_of<N, MULTI>(a, inst), sa, P, T, z, K, L, Lb, x, y, Zl, Zg);
                rr += j;
                k++;
                if ((es > kSSTol) && (k < kSSMaxIt)) {
                    if (k >= a.park_at) {
                        unsigned slot = atomicAdd(a.dst_count, 1u);
                        a.dst.cell[slot] = c;
                        a.dst.k[slot] = k;
                        a.dst.rr[slot] = rr;
                        a.dst.Lb[slot] = Lb;
#pragma unroll
                        for (int i = 0; i < N; i++) a.dst.K[(long)i * a.dst.cap + slot] = K[i];
                        mode = kFetch;
                    } else {
                        L = 0.6;
                        j = 0;
                        big = rr_bound<N>(K);
                        mode = kNewton;
                    }
                } else {
                    flash_store<N>(io, c, L, x, y, Zl, Zg, k, rr);
                    mode = kFetch;
                }
            }
        }
    }
}

template <int N, bool MULTI>
__global__ void __launch_bounds__(128, OSR_FLASH_MIN_BLOCKS) flash_queue_kernel(const __grid_constant__ QueueArgs<N> a) {
    queue_pass<N, MULTI>(a);
}

// ---------------------------------------------------------------------------
// Pair form: two lanes per cell, one per phase.
//
// After the first passes only a few percent of the cells are still
// iterating, and they run for tens to hundreds of substitution steps: the
// late passes leave most of the GPU idle and last as long as the slowest
// cells' steps take one after another.  There the two lanes of a pair
// (lanes 2q and 2q+1 of a warp, `par` = lane & 1) split every step: the
// Rachford-Rice sums and the K update by component parity, the phase work
// (mixing rule, cubic root, logarithms, ln phi) by phase -- lane 0 the
// liquid, lane 1 the vapour -- with xor-1 shuffles between the halves.  Both
// lanes hold K, z and L, and every exchanged value comes out identical in
// the two lanes, so a pair's control flow stays uniform.  The arithmetic is
// the thread-per-cell form's operation for operation; only the order of the
// Rachford-Rice sums differs (each lane sums its components, then the two
// halves are added).

constexpr unsigned kPairFull = 0xffffffffu;

// (value of component 2k + par) for the half arrays of a lane; `pad` for the
// odd lane's missing last component when N is odd.
template <int N>
__device__ __forceinline__ double half_pick(const double *a, int k, int par, double pad) {
    const double e = a[2 * k];
    const double o = (2 * k + 1 < N) ? a[2 * k + 1] : pad;
    return par ? o : e;
}

template <int N>
__device__ __forceinline__ void pair_halves(const double *K, const double *z, int par, double *Kh, double *zh) {
#pragma unroll
    for (int k = 0; k < (N + 1) / 2; k++) {
        Kh[k] = half_pick<N>(K, k, par, 1.0);
        zh[k] = half_pick<N>(z, k, par, 0.0);
    }
}

// One Rachford-Rice Newton step over this lane's components (K, z of the
// components 2k + par; a pad component has K = 1, z = 0 and adds nothing),
// the halves summed across the pair.  `mask` = the lanes taking the step.
template <int N, bool Fast>
__device__ __forceinline__ double rr_step_pair_impl(const double *Kh, const double *zh, double L, bool &ok,
                                                    unsigned mask) {
    constexpr int H = (N + 1) / 2;
    double zt = 0, zq = 0;
    const double omL = 1 - L;
#pragma unroll
    for (int k = 0; k < H; k++) {
        const bool pos = Kh[k] >= 0;
        double num = pos ? 1 - Kh[k] : 1.0;
        double den = pos ? L + omL * Kh[k] : L - 1;
        double td;
        if (Fast) {
            ok &= qdiv_ok(num, den);
            td = qdiv(num, den);
        } else {
            td = num / den;
        }
        const double a = zh[k] * td;
        zt += a;
        zq += a * td;
    }
    const double F = zt + __shfl_xor_sync(mask, zt, 1), dF = -(zq + __shfl_xor_sync(mask, zq, 1));
    double t;
    if (Fast) {
        ok &= qdiv_ok(F, dF);
        t = qdiv(F, dF);
    } else {
        t = F / dF;
    }
    return t;
}

template <int N>
__device__ __forceinline__ double rr_step_pair(const double *Kh, const double *zh, double &L, unsigned mask) {
    bool ok = true;
    double t = rr_step_pair_impl<N, true>(Kh, zh, L, ok, mask);
    ok = __shfl_xor_sync(mask, (int)ok, 1) && ok;
    // pairs with an out-of-range operand redo the step with IEEE division
    const unsigned redo = __ballot_sync(mask, !ok);
    if (redo && !ok) {
        bool ok2 = true;
        t = rr_step_pair_impl<N, false>(Kh, zh, L, ok2, redo);
    }
    L -= t;
    return t;
}

// One substitution step (as ss_update_impl), split across the pair.  x, y,
// Zl, Zg and Kn come out identical in both lanes.  `mask` = the lanes taking
// the step.
template <int N, bool Fast>
__device__ __forceinline__ double ss_update_pair_impl(const FluidTable<N> &f, const double *sa, double P, double T,
                                                      const double *z, const double *K, double *Kn, double L0,
                                                      double &L, double Lb, double *x, double *y, double &Zl,
                                                      double &Zg, bool &ok, int par, unsigned mask) {
    constexpr int H = (N + 1) / 2;
    auto DIV = [&](double a, double b) -> double {
        if (Fast) {
            ok &= qdiv_ok(a, b);
            return qdiv(a, b);
        }
        return a / b;
    };
    L = L0;
    if (L > 1) L = 1;
    else if (L < 0) L = 0;
    const double es = fabs(Lb - L);
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (K[i] >= 0) {
            x[i] = DIV(z[i], L + K[i] * (1 - L));
            y[i] = K[i] * x[i];
        } else {
            x[i] = 0;
            y[i] = DIV(z[i], 1 - L);
        }
    }
    // this lane's phase
    double u[N], v[N];
#pragma unroll
    for (int i = 0; i < N; i++) u[i] = (par ? y[i] : x[i]) * sa[i];
    double Ca = 0, Cb = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < N; j++) s += f.bic[i * N + j] * u[j];
        v[i] = s;
        Ca += u[i] * s;
        Cb += (par ? y[i] : x[i]) * f.b[i];
    }
    const double pa = P / (kR * kR * T * T), pb = P / (kR * T);
    const double A = Ca * pa, B = Cb * pb;
    const bool srk = f.srk != 0;
    const double Z = phase_z(A, B, srk, par != 0);
    const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
    const double DD = DIV(A, B * (d1 - d2));
    const double FF = log(DIV(Z + d2 * B, Z + d1 * B));
    const double cz = log(Z - B);
    const double rCa = DIV(2.0, Ca), rCb = DIV(1.0, Cb);
    const double DF = DD * FF;
    double ln[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        const double t1 = f.b[i] * rCb;
        ln[i] = t1 * (Z - 1) - cz + DF * (sa[i] * v[i] * rCa - t1);
    }
    const double Zo = __shfl_xor_sync(mask, Z, 1);
    Zl = par ? Zo : Z;
    Zg = par ? Z : Zo;
    // K update: this lane takes the components 2k + par and needs the other
    // phase's ln phi of exactly those components
    double Kh[H];
#pragma unroll
    for (int k = 0; k < H; k++) {
        const int ie = 2 * k, io = 2 * k + 1 < N ? 2 * k + 1 : 2 * k;
        const double send = par ? ln[ie] : ln[io];
        const double recv = __shfl_xor_sync(mask, send, 1);
        const double lnl = par ? recv : ln[ie];
        const double lng = par ? ln[io] : recv;
        const double Kk = par ? K[io] : K[ie], xk = par ? x[io] : x[ie], yk = par ? y[io] : y[ie];
        const double zk = (par && 2 * k + 1 >= N) ? 0.0 : (par ? z[io] : z[ie]);
        const double d = lnl - lng;
        const bool fast = Kk > 0 && xk > 0 && yk > 0 && xk < 1e300 && yk < 1e300 && fabs(lnl) < 700 &&
                          fabs(lng) < 700 && fabs(d) < 700;
        const double e = exp(fast ? d : 0.0);
        double kn = (zk != 0 && fast) ? e : Kk;
        if (!(fast || zk == 0)) {
            const double fL = xk * exp(lnl), fG = yk * exp(lng);
            if (fG != 0) kn = Kk * (fL / fG);
            else kn = -1;
            if (fL != fL) kn = -1;
            if (fG != fG) kn = 1;
        }
        Kh[k] = kn;
    }
#pragma unroll
    for (int k = 0; k < H; k++) {
        const double other = __shfl_xor_sync(mask, Kh[k], 1);
        Kn[2 * k] = par ? other : Kh[k];
        if (2 * k + 1 < N) Kn[2 * k + 1] = par ? Kh[k] : other;
    }
    return es;
}

template <int N>
__device__ __forceinline__ double ss_update_pair(const FluidTable<N> &f, const double *sa, double P, double T,
                                                 const double *z, double *K, double &L, double &Lb, double *x,
                                                 double *y, double &Zl, double &Zg, int par, unsigned mask) {
    bool ok = true;
    double Kn[N];
    const double L0 = L;
    double es = ss_update_pair_impl<N, true>(f, sa, P, T, z, K, Kn, L0, L, Lb, x, y, Zl, Zg, ok, par, mask);
    ok = __shfl_xor_sync(mask, (int)ok, 1) && ok;
    const unsigned redo = __ballot_sync(mask, !ok);
    if (redo && !ok) {
        bool ok2 = true;
        es = ss_update_pair_impl<N, false>(f, sa, P, T, z, K, Kn, L0, L, Lb, x, y, Zl, Zg, ok2, par, redo);
    }
#pragma unroll
    for (int i = 0; i < N; i++) K[i] = Kn[i];
    Lb = L;
    return es;
}

// Batched pair form: the queue kernel's passes with two lanes per cell
// (used for the late passes, on the cells parked by the earlier ones).
template <int N, bool MULTI>
__device__ __forceinline__ void pair_pass(const QueueArgs<N> &a) {
    constexpr int H = (N + 1) / 2;
    const int lane = threadIdx.x & 31;
    const int par = lane & 1;
    const FlashIO &io = a.io;
    const long total = a.first ? io.n : (long)__ldcg(a.src_count);
    int mode = kFetch;
    long c = -1;
    double P = 0, T = 0, L = 0, Lb = 10;
    double z[N], K[N], sa[N], Kh[H], zh[H];
    int j = 0, k = 0, rr = 0;
    int waited = 0;
    int inst = 0;
    double big = 0;
#pragma unroll
    for (int i = 0; i < N; i++) z[i] = K[i] = sa[i] = 0;
#pragma unroll
    for (int q = 0; q < H; q++) Kh[q] = zh[q] = 0;
    for (;;) {
        // one slot per pair, claimed through its even lane
        const unsigned need = __ballot_sync(kPairFull, mode == kFetch && par == 0);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(a.head, (unsigned long long)__popc(need));
            base = __shfl_sync(kPairFull, base, leader);
            // both lanes of a pair count the even lanes below the pair: same slot
            const long q = (long)base + __popc(need & ((1u << (lane & ~1)) - 1));
            if (mode == kFetch) {
                if (q < total) {
                    if (a.first) {
                        c = q;
                        k = 0;
                        rr = 0;
                        Lb = 10;
                    } else {
                        c = __ldcg(a.src.cell + q);
                        k = __ldcg(a.src.k + q);
                        rr = __ldcg(a.src.rr + q);
                        Lb = __ldcg(a.src.Lb + q);
#pragma unroll
                        for (int i = 0; i < N; i++) K[i] = __ldcg(a.src.K + (long)i * a.src.cap + q);
                    }
                    P = io.P[c];
                    T = io.T[c];
#pragma unroll
                    for (int i = 0; i < N; i++) z[i] = io.z[(long)i * io.n + c];
                    if constexpr (MULTI) inst = find_instance(a.inst_start, a.n_inst, c);
                    if (a.first) flash_init<N>(table_of<N, MULTI>(a, inst), P, T, K, sa);
                    else sqrt_a<N>(table_of<N, MULTI>(a, inst), T, sa);
                    pair_halves<N>(K, z, par, Kh, zh);
                    L = 0.6;
                    j = 0;
                    big = rr_bound<N>(K);
                    mode = kNewton;
                } else {
                    mode = kDone;
                }
            }
        }
        if (__ballot_sync(kPairFull, mode != kDone) == 0) break;
        const unsigned newton = __ballot_sync(kPairFull, mode == kNewton);
        if (mode == kNewton) {
            const double t = rr_step_pair<N>(Kh, zh, L, newton);
            j++;
            if (fabs(L) > big) {
                j = kRRMaxIt;  // provably divergent: the reference runs to its cap
                mode = kReady;
            } else if (!((t * t > kRRTol) && (j < kRRMaxIt))) {
                mode = kReady;
            }
        }
        const unsigned ready = __ballot_sync(kPairFull, mode == kReady);
        const unsigned still = __ballot_sync(kPairFull, mode == kNewton);
        if (ready != 0) waited++;
        if (ready != 0 && (__popc(ready) >= a.ss_batch || still == 0 || waited > a.max_wait)) {
            waited = 0;
            if (mode == kReady) {
                double x[N], y[N], Zl, Zg;
                const double es = ss_update_pair<N>(table_of<N, MULTI>(a, inst), sa, P, T, z, K, L, Lb, x, y, Zl,
                                                    Zg, par, ready);
                rr += j;
                k++;
                if ((es > kSSTol) && (k < kSSMaxIt)) {
                    if (k >= a.park_at) {
                        if (par == 0) {
                            const unsigned slot = atomicAdd(a.dst_count, 1u);
                            a.dst.cell[slot] = c;
                            a.dst.k[slot] = k;
                            a.dst.rr[slot] = rr;
                            a.dst.Lb[slot] = Lb;
#pragma unroll
                            for (int i = 0; i < N; i++) a.dst.K[(long)i * a.dst.cap + slot] = K[i];
                        }
                        mode = kFetch;
                    } else {
                        pair_halves<N>(K, z, par, Kh, zh);
                        L = 0.6;
                        j = 0;
                        big = rr_bound<N>(K);
                        mode = kNewton;
                    }
                } else {
                    if (par == 0) {
                        io.label[c] = flash_label(L);
                        io.L[c] = L;
#pragma unroll
                        for (int i = 0; i < N; i++) io.x[(long)i * io.n + c] = x[i];
                        io.Zl[c] = Zl;
                        if (io.iters) io.iters[c] = k;
                        if (io.rr_iters) io.rr_iters[c] = rr;
                    } else {
#pragma unroll
                        for (int i = 0; i < N; i++) io.y[(long)i * io.n + c] = y[i];
                        io.Zg[c] = Zg;
                    }
                    mode = kFetch;
                }
            }
        }
    }
}

template <int N, bool MULTI>
__global__ void __launch_bounds__(128, OSR_FLASH_MIN_BLOCKS) flash_pair_kernel(const __grid_constant__ QueueArgs<N> a) {
    pair_pass<N, MULTI>(a);
}

// ---------------------------------------------------------------------------
// Group form: G lanes per cell (G = 4, 8 or 16 lanes, at least N), for the
// last passes, where a few thousand cells run their last hundreds of
// substitution steps with most of the GPU idle and each step's length is set
// by the instructions one lane executes.  Lane r of a group owns component r
// (lanes r >= N hold zero padding): its compositions, its row of the mixing
// rule (the other components' w_j sqrt(a_j) come by shuffle), its ln phi in
// both phases and its K update; the sums over components are butterfly
// reductions, which leave the same value in every lane of the group; the
// two phases' cubic roots, logarithms and quotients run on alternate lanes
// and are exchanged.  The Rachford-Rice Newton run is replicated in every
// lane (all K and z are kept in every lane), so it is the thread-per-cell
// form's arithmetic exactly.  Only the order of the mixing and b sums
// differs from the thread-per-cell form (a tree instead of a running sum).

template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// One substitution step of a group (as ss_update_impl).  Per lane: xi, yi,
// Kn of its own component; Zl, Zg identical in the group.  `bic` = the
// lane's row of 1 - k_ij, sai / bi its sqrt(a) and b (zero for pad lanes).
template <int N, int G, bool Fast>
__device__ __forceinline__ double ss_update_group_impl(const double *bic, double sai, double bi, bool srk, double P,
                                                       double T, double zi, double Ki, double L0, double &L,
                                                       double Lb, double &xi, double &yi, double &Zl, double &Zg,
                                                       double &Kn, bool &ok, int r, int base, unsigned mask) {
    auto DIV = [&](double a, double b) -> double {
        if (Fast) {
            ok &= qdiv_ok(a, b);
            return qdiv(a, b);
        }
        return a / b;
    };
    L = L0;
    if (L > 1) L = 1;
    else if (L < 0) L = 0;
    const double es = fabs(Lb - L);
    const bool own = r < N;
    xi = 0;
    yi = 0;
    if (own) {
        if (Ki >= 0) {
            xi = DIV(zi, L + Ki * (1 - L));
            yi = Ki * xi;
        } else {
            yi = DIV(zi, 1 - L);
        }
    }
    const double ul = xi * sai, ug = yi * sai;
    double vl = 0, vg = 0;
#pragma unroll
    for (int j = 0; j < N; j++) {
        const double ulj = __shfl_sync(mask, ul, base + j), ugj = __shfl_sync(mask, ug, base + j);
        vl += bic[j] * ulj;
        vg += bic[j] * ugj;
    }
    const double Cal = group_sum<G>(ul * vl, mask), Cag = group_sum<G>(ug * vg, mask);
    const double Cbl = group_sum<G>(xi * bi, mask), Cbg = group_sum<G>(yi * bi, mask);
    // this lane's phase for the scalar work: even lanes liquid, odd vapour
    const int p = r & 1;
    const double pa = P / (kR * kR * T * T), pb = P / (kR * T);
    const double Ca = p ? Cag : Cal, Cb = p ? Cbg : Cbl;
    const double A = Ca * pa, B = Cb * pb;
    const double Z = phase_z(A, B, srk, p != 0);
    const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
    const double DD = DIV(A, B * (d1 - d2));
    const double FF = log(DIV(Z + d2 * B, Z + d1 * B));
    const double cz = log(Z - B);
    const double rCa = DIV(2.0, Ca), rCb = DIV(1.0, Cb);
    const double DF = DD * FF;
    const double Zo = __shfl_xor_sync(mask, Z, 1), DFo = __shfl_xor_sync(mask, DF, 1);
    const double czo = __shfl_xor_sync(mask, cz, 1), rCao = __shfl_xor_sync(mask, rCa, 1);
    const double rCbo = __shfl_xor_sync(mask, rCb, 1);
    Zl = p ? Zo : Z;
    Zg = p ? Z : Zo;
    const double DFl = p ? DFo : DF, DFg = p ? DF : DFo, cl = p ? czo : cz, cg = p ? cz : czo;
    const double rCal = p ? rCao : rCa, rCag = p ? rCa : rCao, rCbl = p ? rCbo : rCb, rCbg = p ? rCb : rCbo;
    Kn = Ki;
    if (own) {
        const double t1l = bi * rCbl, t1g = bi * rCbg;
        const double lnl = t1l * (Zl - 1) - cl + DFl * (sai * vl * rCal - t1l);
        const double lng = t1g * (Zg - 1) - cg + DFg * (sai * vg * rCag - t1g);
        const double d = lnl - lng;
        const bool fast = Ki > 0 && xi > 0 && yi > 0 && xi < 1e300 && yi < 1e300 && fabs(lnl) < 700 &&
                          fabs(lng) < 700 && fabs(d) < 700;
        const double e = exp(fast ? d : 0.0);
        Kn = (zi != 0 && fast) ? e : Ki;
        if (!(fast || zi == 0)) {
            const double fL = xi * exp(lnl), fG = yi * exp(lng);
            if (fG != 0) Kn = Ki * (fL / fG);
            else Kn = -1;
            if (fL != fL) Kn = -1;
            if (fG != fG) Kn = 1;
        }
    }
    return es;
}

template <int N, int G>
__device__ __forceinline__ double ss_update_group(const double *bic, double sai, double bi, bool srk, double P,
                                                  double T, double zi, double &Ki, double *K, double &L, double &Lb,
                                                  double &xi, double &yi, double &Zl, double &Zg, int r, int base,
                                                  unsigned mask) {
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1)) << base;
    bool ok = true;
    double Kn;
    const double L0 = L;
    double es = ss_update_group_impl<N, G, true>(bic, sai, bi, srk, P, T, zi, Ki, L0, L, Lb, xi, yi, Zl, Zg, Kn, ok,
                                                 r, base, mask);
    // a group with an out-of-range operand in any lane redoes the step with
    // IEEE division
    const unsigned bad = __ballot_sync(mask, !ok);
    const unsigned redo = __ballot_sync(mask, (bad & gmask) != 0);
    if (redo && (bad & gmask)) {
        bool ok2 = true;
        es = ss_update_group_impl<N, G, false>(bic, sai, bi, srk, P, T, zi, Ki, L0, L, Lb, xi, yi, Zl, Zg, Kn, ok2,
                                               r, base, redo);
    }
    Ki = Kn;
#pragma unroll
    for (int j = 0; j < N; j++) K[j] = __shfl_sync(mask, Kn, base + j);
    Lb = L;
    return es;
}

// Batched group form: the queue kernel's passes with G lanes per cell (used
// for the last passes, on the cells parked by the earlier ones).
template <int N, int G, bool MULTI>
__global__ void __launch_bounds__(128) flash_group_kernel(const __grid_constant__ QueueArgs<N> a) {
    static_assert(G >= N && G >= 2 && (G & (G - 1)) == 0 && G <= 32, "G lanes per cell, a power of two >= N");
    const int lane = threadIdx.x & 31;
    const int r = lane & (G - 1), base = lane & ~(G - 1);
    const FlashIO &io = a.io;
    const long total = a.first ? io.n : (long)__ldcg(a.src_count);
    int mode = kFetch;
    long c = -1;
    double P = 0, T = 0, L = 0, Lb = 10;
    double z[N], K[N], bic[N];
    double sai = 0, bi = 0, zi = 0, Ki = 0;
    bool srk = false;
    int j = 0, k = 0, rr = 0;
    int waited = 0;
    int inst = 0;
    double big = 0;
#pragma unroll
    for (int i = 0; i < N; i++) z[i] = K[i] = bic[i] = 0;
    for (;;) {
        // one slot per group, claimed through its first lane
        const unsigned need = __ballot_sync(kPairFull, mode == kFetch && r == 0);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned long long slot0 = 0;
            if (lane == leader) slot0 = atomicAdd(a.head, (unsigned long long)__popc(need));
            slot0 = __shfl_sync(kPairFull, slot0, leader);
            const long q = (long)slot0 + __popc(need & ((1u << base) - 1));
            if (mode == kFetch) {
                if (q < total) {
                    if (a.first) {
                        c = q;
                        k = 0;
                        rr = 0;
                        Lb = 10;
                    } else {
                        c = __ldcg(a.src.cell + q);
                        k = __ldcg(a.src.k + q);
                        rr = __ldcg(a.src.rr + q);
                        Lb = __ldcg(a.src.Lb + q);
#pragma unroll
                        for (int i = 0; i < N; i++) K[i] = __ldcg(a.src.K + (long)i * a.src.cap + q);
                    }
                    P = io.P[c];
                    T = io.T[c];
#pragma unroll
                    for (int i = 0; i < N; i++) z[i] = io.z[(long)i * io.n + c];
                    if constexpr (MULTI) inst = find_instance(a.inst_start, a.n_inst, c);
                    const FluidTable<N> &f = table_of<N, MULTI>(a, inst);
                    double sa[N];
                    if (a.first) flash_init<N>(f, P, T, K, sa);
                    else sqrt_a<N>(f, T, sa);
                    // this lane's component (zero padding past N)
                    sai = bi = zi = 0;
                    Ki = 1;
#pragma unroll
                    for (int i = 0; i < N; i++)
                        if (i == r) {
                            sai = sa[i];
                            bi = f.b[i];
                            zi = z[i];
                            Ki = K[i];
                        }
#pragma unroll
                    for (int jj = 0; jj < N; jj++) bic[jj] = r < N ? f.bic[(r < N ? r : 0) * N + jj] : 0.0;
                    srk = f.srk != 0;
                    L = 0.6;
                    j = 0;
                    big = rr_bound<N>(K);
                    mode = kNewton;
                } else {
                    mode = kDone;
                }
            }
        }
        if (__ballot_sync(kPairFull, mode != kDone) == 0) break;
        if (mode == kNewton) {
            const double t = rr_step<N>(K, z, L);
            j++;
            if (fabs(L) > big) {
                j = kRRMaxIt;  // provably divergent: the reference runs to its cap
                mode = kReady;
            } else if (!((t * t > kRRTol) && (j < kRRMaxIt))) {
                mode = kReady;
            }
        }
        const unsigned ready = __ballot_sync(kPairFull, mode == kReady);
        const unsigned still = __ballot_sync(kPairFull, mode == kNewton);
        if (ready != 0) waited++;
        if (ready != 0 && (__popc(ready) >= a.ss_batch || still == 0 || waited > a.max_wait)) {
            waited = 0;
            if (mode == kReady) {
                double xi, yi, Zl, Zg;
                const double es = ss_update_group<N, G>(bic, sai, bi, srk, P, T, zi, Ki, K, L, Lb, xi, yi, Zl, Zg, r,
                                                        base, ready);
                rr += j;
                k++;
                // es and k are the same in every lane of a group
                const bool go_on = (es > kSSTol) && (k < kSSMaxIt);
                const unsigned parkers = __ballot_sync(ready, go_on && k >= a.park_at);
                if (go_on) {
                    if (k >= a.park_at) {
                        unsigned slot = 0;
                        if (r == 0) slot = atomicAdd(a.dst_count, 1u);
                        slot = __shfl_sync(parkers, slot, base);
                        if (r == 0) {
                            a.dst.cell[slot] = c;
                            a.dst.k[slot] = k;
                            a.dst.rr[slot] = rr;
                            a.dst.Lb[slot] = Lb;
                        }
                        if (r < N) a.dst.K[(long)r * a.dst.cap + slot] = Ki;
                        mode = kFetch;
                    } else {
                        L = 0.6;
                        j = 0;
                        big = rr_bound<N>(K);
                        mode = kNewton;
                    }
                } else {
                    if (r < N) {
                        io.x[(long)r * io.n + c] = xi;
                        io.y[(long)r * io.n + c] = yi;
                    }
                    if (r == 0) {
                        io.label[c] = flash_label(L);
                        io.L[c] = L;
                        io.Zl[c] = Zl;
                        io.Zg[c] = Zg;
                        if (io.iters) io.iters[c] = k;
                        if (io.rr_iters) io.rr_iters[c] = rr;
                    }
                    mode = kFetch;
                }
            }
        }
    }
}

// Lanes per cell of the group form for N components.
template <int N>
constexpr int group_lanes() {
    return N <= 2 ? 2 : N <= 4 ? 4 : N <= 8 ? 8 : 16;
}

// Fugacity derivatives for both phases of every cell, following the
// reference's fugacity rows of the analytic Jacobian
// (compsim/Petsc_Functions.cpp:30243-30372) with dZ/dP, dZ/dw_k from the
// implicit derivative of the cubic (compsim/Do_Cycle.cpp:517-552):
//   dlnphi_dx[ph][i][k][c] = d ln phi_i / d w_k,  dlnphi_dP[ph][i][c].
template <int N>
struct DerivArgs {
    FluidTable<N> f;
    const double *P, *T, *x, *y, *Zl, *Zg;
    long n;
    double *dlnphi_dx, *dlnphi_dP;
    const FluidTable<N> *tables;   // several instances (see QueueArgs)
    const long *inst_start;
    int n_inst;
};

// store_dx(i, k, value) receives d ln(phi_i)/d w_k, store_dp(i, value)
// d ln(phi_i)/d P.
template <int N, class SX, class SP>
__device__ __forceinline__ void phase_derivs_into(const FluidTable<N> &f, const double *sa, double P, double T,
                                                  const double *w, double Z, SX store_dx, SP store_dp) {
    double u[N], v[N];
#pragma unroll
    for (int i = 0; i < N; i++) u[i] = w[i] * sa[i];
    double Ca = 0, Cb = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < N; j++) s += f.bic[i * N + j] * u[j];
        v[i] = s;  // sum_j w_j sqrt(a_i a_j)(1-k_ij) = sa[i] * v[i]
        Ca += u[i] * s;
        Cb += w[i] * f.b[i];
    }
    const bool srk = f.srk != 0;
    const double rt = kR * T;
    const double pa = P / (rt * rt), pb = P / rt;
    double A = Ca * pa, B = Cb * pb;
    double dAdp = Ca / (rt * rt), dBdp = Cb / rt;
    double U = srk ? B : 2 * B, W = srk ? 0.0 : B;
    double dUdp = srk ? dBdp : 2 * dBdp, dWdp = srk ? 0.0 : dBdp;
    const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
    double rden = 1 / (3 * Z * Z - 2 * Z * (1 + B - U) + A - B * U - U - W * W);
    // coefficients of the implicit derivative dZ = -(cA dA + cB dB + cU dU + cW dW)/den
    double cA = Z - B, cB = -Z * Z - U * Z - A + W * W, cU = Z * Z - B * Z - Z, cW = -2 * W * Z + 2 * B * W + 2 * W;
    double dZdp = -(dAdp * cA + dBdp * cB + dUdp * cU + dWdp * cW) * rden;
    double DD = A / (B * (d1 - d2));
    double FF = log((Z + d2 * B) / (Z + d1 * B));
    double rZB = 1 / (Z - B), rZ1 = 1 / (Z + d1 * B), rZ2 = 1 / (Z + d2 * B);
    double rCa = 1 / Ca, rCb = 1 / Cb;
    double dDDdp = (B * dAdp - A * dBdp) / (B * B * (d1 - d2));
    double dFFdp = (dZdp + d2 * dBdp) * rZ2 - (dZdp + d1 * dBdp) * rZ1;
    double dBBdp = (dBdp - dZdp) * rZB;
    // Per-k factors of d ln(phi_i)/d w_k.  Expanding the reference's
    //   dAA + dBB + dDD EE FF + DD dEE FF + DD EE dFF
    // with dAA = -b_k t1 (Z-1)/Cb + t1 dZ_k, dBB = (dB_k - dZ_k)/(Z-B),
    // dEE = 2 a_ik/Ca - 2 t_i dA_k/(pa Ca^2) + t1 b_k/Cb  (t1 = b_i/Cb) gives
    //   t1 P1_k + P2_k + EE P3_k + (2 DD FF/Ca) a_ik - g_i P4_k.
    double P1[N], P2[N], P3[N], P4[N];
    const double twopa = 2 * pa;
    const double rBB = 1 / (B * B * (d1 - d2));
    const double DF = DD * FF;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double dA = sa[k] * v[k] * twopa;
        double dB = f.b[k] * pb;
        double dU = srk ? dB : 2 * dB, dW = srk ? 0.0 : dB;
        double dZ = -(dA * cA + dB * cB + dU * cU + dW * cW) * rden;
        double dDD = (dA * B - dB * A) * rBB;
        double dFF = (dZ + d2 * dB) * rZ2 - (dZ + d1 * dB) * rZ1;
        P1[k] = dZ - f.b[k] * (Z - 1) * rCb + DF * f.b[k] * rCb;
        P2[k] = (dB - dZ) * rZB;
        P3[k] = dDD * FF + DD * dFF;
        P4[k] = DF * dA;
    }
    const double rpa = 1 / pa;
    const double h = 2 * DF * rCa;
#pragma unroll 1
    for (int i = 0; i < N; i++) {
        double sai = 0, vi = 0, bi = 0;
        // select sa[i], v[i], b[i] without dynamic register indexing
#pragma unroll
        for (int q = 0; q < N; q++)
            if (q == i) { sai = sa[q]; vi = v[q]; bi = f.b[q]; }
        double ti = sai * vi;
        double t1 = bi * rCb;
        double EE = 2 * ti * rCa - t1;
        store_dp(i, t1 * dZdp + dBBdp + EE * (dDDdp * FF + DD * dFFdp));
        double g = 2 * ti * rCa * rCa * rpa;
        double hs = h * sai;
#pragma unroll
        for (int k = 0; k < N; k++) {
            store_dx(i, k, t1 * P1[k] + P2[k] + EE * P3[k] + hs * sa[k] * f.bic[i * N + k] - g * P4[k]);
        }
    }
}

template <int N>
__device__ __forceinline__ void phase_derivs(const FluidTable<N> &f, const double *sa, double P, double T,
                                             const double *w, double Z, double *out_dx, double *out_dp, long n,
                                             long c) {
    phase_derivs_into<N>(
        f, sa, P, T, w, Z, [&](int i, int k, double v) { out_dx[((long)i * N + k) * n + c] = v; },
        [&](int i, double v) { out_dp[(long)i * n + c] = v; });
}

// One thread per (cell, phase); blockIdx.y selects the phase.
// Cells c0, c0 + stride, ... below c1 of phase ph.  The phase compositions
// and Z factors are read through L2 (a persistent launch reads what other
// CTAs wrote earlier in the same launch).
template <int N, bool MULTI>
__device__ __forceinline__ void deriv_cells(const DerivArgs<N> &a, int ph, long c0, long c1, long stride) {
    const double *comp = ph ? a.y : a.x;
    const double *Zp = ph ? a.Zg : a.Zl;
    double *odx = a.dlnphi_dx + (long)ph * N * N * a.n;
    double *odp = a.dlnphi_dP + (long)ph * N * a.n;
    for (long c = c0; c < c1; c += stride) {
        double sa[N], w[N];
        double T = a.T[c];
        int inst = 0;
        if constexpr (MULTI) inst = find_instance(a.inst_start, a.n_inst, c);
        const FluidTable<N> &f = table_of<N, MULTI>(a, inst);
        sqrt_a<N>(f, T, sa);
#pragma unroll
        for (int i = 0; i < N; i++) w[i] = __ldcg(comp + (long)i * a.n + c);
        phase_derivs<N>(f, sa, a.P[c], T, w, __ldcg(Zp + c), odx, odp, a.n, c);
    }
}

template <int N, bool MULTI>
__global__ void __launch_bounds__(128) flash_deriv_kernel(const __grid_constant__ DerivArgs<N> a) {
    deriv_cells<N, MULTI>(a, blockIdx.y, (long)blockIdx.x * blockDim.x + threadIdx.x, a.n,
                          (long)gridDim.x * blockDim.x);
}

}  // namespace osr
