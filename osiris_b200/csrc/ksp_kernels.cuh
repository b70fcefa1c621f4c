// Device linear solve of the Newton system on the compact Jacobian: the
// reference's PETSc configuration (SolveNonLinear, compsim/PetscAUX.cpp:
// 631-646: KSPSetType(SolverType = "bcgs"), PCSetType(PCVPBJACOBI) with the
// PJac block sizes, KSPSetTolerances(RELTOL, ABSTOL, DIVTOL, MAXITERS)).
//
// PETSc is a third-party dependency the reference links against and does not
// ship; its algorithms are restated here from their published form:
//  * BiCGStab (van der Vorst, SIAM J. Sci. Stat. Comput. 13, 1992) in PETSc's
//    left-preconditioned arrangement (KSPBCGS): zero initial guess, the
//    preconditioned residual r = B (b - A x) and its 2-norm drive the
//    convergence test, the shadow residual is r_0, breakdown when
//    (v, r_0) = 0, when t = 0 with s != 0, or when rho = 0.
//  * KSPConvergedDefault: ttol = max(rtol |r_0|, atol); converged when
//    |r_k| <= ttol (ATOL when |r_k| < atol, else RTOL), diverged when
//    |r_k| >= dtol |r_0|, or when a norm or dot product is not finite;
//    DIVERGED_ITS after max_it iterations.
//  * PCVPBJACOBI: the inverse of every variable-size diagonal block (one
//    block per cell-medium, 2N+4 or N+3 rows), applied block by block.
// Reason codes are PETSc's KSPConvergedReason values.
//
// Kernels, per iteration (each returns at once when the solve has ended,
// so the host may enqueue iterations in batches and poll the status rarely):
//   bcgs_p       p <- r + beta (p - omega_old v)
//   spmv         t <- A p                  (two or four lanes per block row)
//   bjac_apply   v <- B t, (v, r0)         (one thread per block row) -> alpha
//   bcgs_s       s <- r - alpha v
//   spmv         w <- A s
//   bjac_apply   t <- B w, (s,t) (t,t) (s,s)                        -> omega
//   bcgs_xr      x += alpha p + omega s, r <- s - omega t, |r|^2, (r, r0)
//                                                      -> test, rho, beta
// Reductions are deterministic: fixed grids, per-CTA partial sums in a fixed
// order, reduced by the last CTA to finish (atomic ticket).
#pragma once
#include <cuda_runtime.h>
#include "jacobian_kernels.cuh"

namespace osrk {

using osrj::Layout;
using osrj::ref_col;
using osrj::ref_row;
using osrj::value_index;

// PETSc KSPConvergedReason values
enum : int {
    kItersRunning = 0,
    kConvergedRtol = 2,
    kConvergedAtol = 3,
    kDivergedIts = -3,
    kDivergedDtol = -4,
    kDivergedBreakdown = -5,
    kDivergedNanOrInf = -9,
    kDivergedPcFailed = -11,
    kFinishWithP = -100,   // internal: t = s = 0, the update is x += alpha p
};

constexpr int kMaxRedBlocks = 148 * 64;   // CTAs of a reducing kernel (partials buffer size)
constexpr int kRedThreads = 256;
constexpr int kParts = 3;         // partial sums per reduction kernel

struct KspScal {
    double rho, rhoold, alpha, omega, omegaold, beta;
    double rnorm0, rnorm, ttol;
    double rtol, atol, dtol;
    int its, max_it, reason, pad;
    unsigned int ticket;
};

struct KView {
    int nc, nx, ny, nz;
    long n;             // cells per continuum
    long rows;          // unknowns
    const long *rowoff; // [2n + 1]
    const signed char *lab_m, *lab_f;
    const double *vals; // compact Jacobian
    int entries;
};

__device__ __forceinline__ int label_of(const KView &v, long b) {
    return b >= v.n ? v.lab_f[b - v.n] : v.lab_m[b];
}

// Target block of slot s of block row b (-1 beyond the grid).
__device__ __forceinline__ long slot_block(const KView &v, long b, int s) {
    const int med = b >= v.n;
    const long c = med ? b - v.n : b;
    const int ix = (int)(c % v.nx), iy = (int)((c / v.nx) % v.ny), iz = (int)(c / ((long)v.nx * v.ny));
    const long sy = v.nx, sz = (long)v.nx * v.ny;
    switch (s) {
        case 0: return b;
        case 1: return ix == 0 ? -1 : b - 1;
        case 2: return ix == v.nx - 1 ? -1 : b + 1;
        case 3: return iy == 0 ? -1 : b - sy;
        case 4: return iy == v.ny - 1 ? -1 : b + sy;
        case 5: return iz == 0 ? -1 : b - sz;
        case 6: return iz == v.nz - 1 ? -1 : b + sz;
        default: return med ? c : v.n + c;
    }
}

// Global column of shifted entry j (0..7) of block row b, or -1
// (osrj::entry_position restated for the overflow entries).
__device__ __forceinline__ long overflow_col(const KView &v, long b, int j) {
    const int N = v.nc;
    const int med = b >= v.n;
    const long c = med ? b - v.n : b;
    const int iy = (int)((c / v.nx) % v.ny), iz = (int)(c / ((long)v.nx * v.ny));
    const int f = j / 4, t = j % 4;
    if (f == 0 ? iy == 0 : iz == 0) return -1;
    const long stride = f == 0 ? (long)v.nx : (long)v.nx * v.ny;
    const int lnb = (med ? v.lab_f : v.lab_m)[c - stride];
    const int nbase = lnb ? -N : 0, reCol4 = lnb ? 1 : 0;
    const int col = nbase + 2 * N + (t == 3 ? 3 - reCol4 : t);
    const long g = v.rowoff[b - stride + 1] + col;
    return (g >= 0 && g < v.rows) ? g : -1;
}

// Entry index of canonical (row r, slot 0, column cc), or -1 when not stored.
__device__ __forceinline__ int own_entry(const Layout &L, int r, int cc) {
    const int N = L.N;
    if (r < N) return cc <= 2 * N ? L.f(r, cc) : -1;
    if (r < 2 * N) return L.cr(r, 0, cc);
    if (r == 2 * N) return (cc == 2 * N || cc == 2 * N + 1) ? L.w(0, cc) : -1;
    return L.k(r, cc);
}

// ---------------------------------------------------------------------------
// y = A x on the compact layout.  LANES (2 or 4) lanes per block row and
// 32 / LANES block rows per warp: lane = (32 / LANES) g + q serves block row
// base + q and target slots g, g + LANES, ... (slot 0 this cell, 1..6 the
// -x, +x, -y, +y, -z, +z neighbours, 7 the other continuum).  Each entry a
// warp reads is then LANES runs of 256 / LANES contiguous bytes (the block
// rows of one slot).
// A lane gathers its target block's unknowns into canonical positions and
// accumulates the block row's canonical rows in registers; the four partial
// rows are summed by a butterfly over the lanes of the same q and stored at
// the reference-local rows (no atomics: every entry of a block row lies in
// that block row's rows).  The own-slot lane also takes the fugacity and
// constraint rows, the -y and -z lanes the shifted entries of their faces.
// Values whose row the block row does not carry, or whose column the target
// block does not use (one-phase blocks), are not fetched.
// ---------------------------------------------------------------------------
constexpr int kSpmvThreads = 128;
// block rows from which the two-lane form is used
constexpr long kSpmvRowForm = 148L * 2048;

// Up to four components the row and column registers fit a bound of eight
// resident CTAs per SM (64 registers): twice the warps in flight to cover
// the gather and value latency, a pass 13 % faster at 128x128x32 despite a
// few spilled bytes; larger N keeps the compiler's choice.
template <int N, int LANES>
__global__ void __launch_bounds__(kSpmvThreads, (N <= 4 ? 8 : 4)) spmv_kernel(const KView v, const double *__restrict__ x,
                                                             double *__restrict__ y, const KspScal *s) {
    if (s && s->reason != kItersRunning) return;
    static_assert(LANES == 2 || LANES == 4, "two or four lanes per block row");
    constexpr int BS = 2 * N + 4;
    constexpr int ROWS = 32 / LANES;   // block rows per warp
    const Layout L(N);
    const long nb = 2 * v.n;
    const int lane = threadIdx.x & 31, g = lane / ROWS, q = lane % ROWS;
    const long groups = (nb + ROWS - 1) / ROWS;
    const long gstride = (long)gridDim.x * (kSpmvThreads / 32);
    for (long grp = (long)blockIdx.x * (kSpmvThreads / 32) + (threadIdx.x >> 5); grp < groups; grp += gstride) {
        const long b = grp * ROWS + q;
        const bool valid = b < nb;
        double acc[BS];
#pragma unroll
        for (int r = 0; r < BS; r++) acc[r] = 0;
        int lb = 0;
        if (valid) {
            lb = label_of(v, b);
            unsigned long long rm = 0;
#pragma unroll
            for (int r = 0; r < BS; r++) rm |= (unsigned long long)(ref_row(N, lb, r) >= 0) << r;
            const double *val = v.vals + ((b >> 5) * v.entries) * 32 + (b & 31);
#pragma unroll 1
            for (int h = 0; h < 8 / LANES; h++) {
                const int sl = g + LANES * h;
                const long tb = slot_block(v, b, sl);
                if (tb < 0) continue;
                const int lt = label_of(v, tb);
                const long toff = v.rowoff[tb];
                double xs[BS];
                unsigned long long cm = 0;
#pragma unroll
                for (int cc = 0; cc < BS; cc++) {
                    const int rc = ref_col(N, lt, cc);
                    xs[cc] = rc >= 0 ? __ldg(x + toff + rc) : 0.0;
                    cm |= (unsigned long long)(rc >= 0) << cc;
                }
                auto mac = [&](int r, int cc, int e) {
                    if (((rm >> r) & (cm >> cc)) & 1ull) acc[r] += __ldcs(val + 32 * e) * xs[cc];
                };
#pragma unroll
                for (int r = N; r < 2 * N; r++)
#pragma unroll
                    for (int cc = 0; cc < BS; cc++) mac(r, cc, L.cr(r, sl, cc));
                mac(2 * N, 2 * N, L.w(sl, 2 * N));
                mac(2 * N, 2 * N + 1, L.w(sl, 2 * N + 1));
                if (sl == 0) {
#pragma unroll
                    for (int r = 0; r < N; r++)
#pragma unroll
                        for (int cc = 0; cc <= 2 * N; cc++) mac(r, cc, L.f(r, cc));
#pragma unroll
                    for (int r = 2 * N + 1; r < BS; r++)
#pragma unroll
                        for (int cc = 0; cc < BS; cc++) mac(r, cc, L.k(r, cc));
                }
                if ((sl == 3 || sl == 5) && ((rm >> (2 * N - 1)) & 1ull)) {
                    // the shifted entries of the -y (slot 3) and -z (slot 5) faces: columns
                    // counted from the row offset of the block after that neighbour
                    // (osrj::entry_position)
                    const long base = v.rowoff[tb + 1];
                    const int nbase = lt ? -N : 0, reCol4 = lt ? 1 : 0, j0 = sl == 3 ? 0 : 4;
#pragma unroll
                    for (int t = 0; t < 4; t++) {
                        const long gc = base + nbase + 2 * N + (t == 3 ? 3 - reCol4 : t);
                        if (gc >= 0 && gc < v.rows) acc[2 * N - 1] += __ldcs(val + 32 * L.o(j0 + t)) * __ldg(x + gc);
                    }
                }
            }
        }
        // sum the slot lanes of each block row
#pragma unroll
        for (int r = 0; r < BS; r++) {
            double t = acc[r];
#pragma unroll
            for (int o = ROWS; o < 32; o <<= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            acc[r] = t;
        }
        if (valid) {
            const long off = v.rowoff[b];
#pragma unroll
            for (int r = 0; r < BS; r++) {
                if ((r % LANES) != g) continue;
                const int rr = ref_row(N, lb, r);
                if (rr >= 0) y[off + rr] = acc[r];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Block-diagonal inverse, one warp per block row: the diagonal block (the
// own-slot entries, plus any shifted entry whose column falls in the block)
// is assembled in shared memory at reference-local rows and columns and
// inverted in place by Gauss-Jordan elimination with partial pivoting (row
// interchanges undone as column interchanges at the end).  Stored in chunks
// of 32 block rows like the Jacobian values, inv[chunk][j BS + i][32] =
// (A^-1)_ij, so the apply kernel's 32 lanes read 256 contiguous bytes per
// entry.  A zero pivot sets the solve's reason to PC_FAILED.
// ---------------------------------------------------------------------------
constexpr int kInvWarps = 4;

template <int N>
__global__ void __launch_bounds__(32 * kInvWarps) bjac_invert_kernel(const KView v, double *__restrict__ inv,
                                                                      KspScal *s) {
    constexpr int BS = 2 * N + 4;
    __shared__ double sA[kInvWarps][BS * BS];
    __shared__ int sPiv[kInvWarps][BS];
    const Layout L(N);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *A = sA[w];
    int *piv = sPiv[w];
    const long nb = 2 * v.n;
    const long warps = (long)gridDim.x * kInvWarps;
    for (long b = (long)blockIdx.x * kInvWarps + w; b < nb; b += warps) {
        const int lb = label_of(v, b);
        const long off = v.rowoff[b];
        const int bs = (int)(v.rowoff[b + 1] - off);
        const double *val = v.vals + ((b >> 5) * v.entries) * 32 + (b & 31);
        for (int q = lane; q < BS * BS; q += 32) A[q] = (q / BS == q % BS && q / BS >= bs) ? 1.0 : 0.0;
        __syncwarp();
        for (int cc = lane; cc < BS; cc += 32) {
            const int rc = ref_col(N, lb, cc);
            if (rc < 0) continue;
            for (int r = 0; r < BS; r++) {
                const int rr = ref_row(N, lb, r);
                const int e = own_entry(L, r, cc);
                if (rr >= 0 && e >= 0) A[rr * BS + rc] = val[32 * e];
            }
        }
        __syncwarp();
        if (lane == 0) {
            const int rt = ref_row(N, lb, 2 * N - 1);
            for (int j = 0; j < osrj::kOverflow && rt >= 0; j++) {
                const long g = overflow_col(v, b, j);
                if (g >= off && g < off + bs) A[rt * BS + (int)(g - off)] += val[32 * L.o(j)];
            }
        }
        __syncwarp();
        bool singular = false;
        for (int k = 0; k < bs; k++) {
            // pivot: largest |A[i][k]|, i >= k, first index on ties
            double best = -1.0;
            int bi = bs;
            for (int i = k + lane; i < bs; i += 32) {
                const double a = fabs(A[i * BS + k]);
                if (a > best) { best = a; bi = i; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (!(best > 0.0)) { singular = true; break; }
            const int p = bi;
            if (p != k)
                for (int j = lane; j < bs; j += 32) {
                    const double t = A[k * BS + j];
                    A[k * BS + j] = A[p * BS + j];
                    A[p * BS + j] = t;
                }
            if (lane == 0) piv[k] = p;
            __syncwarp();
            const double d = A[k * BS + k];
            __syncwarp();
            for (int j = lane; j < bs; j += 32) A[k * BS + j] = (j == k) ? 1.0 / d : A[k * BS + j] / d;
            __syncwarp();
            for (int j = lane; j < bs; j += 32) {
                if (j == k) continue;
                const double akj = A[k * BS + j];
                for (int i = 0; i < bs; i++)
                    if (i != k) A[i * BS + j] -= A[i * BS + k] * akj;
            }
            __syncwarp();
            const double ikk = A[k * BS + k];
            for (int i = lane; i < bs; i += 32)
                if (i != k) A[i * BS + k] = -A[i * BS + k] * ikk;
            __syncwarp();
        }
        if (singular) {
            if (lane == 0) atomicExch(&s->reason, kDivergedPcFailed);
            __syncwarp();
            continue;
        }
        for (int k = bs - 1; k >= 0; k--) {
            const int p = piv[k];
            if (p != k)
                for (int i = lane; i < bs; i += 32) {
                    const double t = A[i * BS + k];
                    A[i * BS + k] = A[i * BS + p];
                    A[i * BS + p] = t;
                }
            __syncwarp();
        }
        double *o = inv + ((b >> 5) * (BS * BS)) * 32 + (b & 31);
        for (int q = lane; q < BS * BS; q += 32) o[32 * q] = A[(q % BS) * BS + q / BS];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Reductions: per-CTA partial sums (fixed order), the last CTA reduces the
// partials in CTA order and runs the scalar step.
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double *sm) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < K; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; q++) sm[q * 32 + w] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < K; q++) {
            double t = 0;
            for (int i = 0; i < nw; i++) t += sm[q * 32 + i];
            v[q] = t;
        }
}

// Publish this CTA's K partials (part[q][gridDim.x]); returns true in thread
// 0 of the last CTA to finish, with the totals in tot.  The last CTA's
// threads sum fixed strided subsets of the partials, then reduce them as one
// block, so the order never depends on timing.
template <int K>
__device__ bool publish_partials(double (&v)[K], double *part, KspScal *s, double (&tot)[K]) {
    __shared__ double sm[K * 32];
    __shared__ bool last;
    block_sums<K>(v, sm);
    const int nblk = (int)gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) part[q * nblk + blockIdx.x] = v[q];
        __threadfence();
        const unsigned t = atomicAdd(&s->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double w[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
        double t = 0;
        for (int i = threadIdx.x; i < nblk; i += blockDim.x) t += ((volatile double *)part)[q * nblk + i];
        w[q] = t;
    }
    __syncthreads();
    block_sums<K>(w, sm);
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int q = 0; q < K; q++) tot[q] = w[q];
    s->ticket = 0;
    return true;
}

// KSPConvergedDefault on the current residual norm (iteration its).
__device__ __forceinline__ void converged_test(KspScal *s, double rnorm) {
    if (!isfinite(rnorm)) {
        s->reason = kDivergedNanOrInf;
    } else if (rnorm <= s->ttol) {
        s->reason = rnorm < s->atol ? kConvergedAtol : kConvergedRtol;
    } else if (s->its > 0 && s->dtol > 0 && rnorm >= s->dtol * s->rnorm0) {
        s->reason = kDivergedDtol;
    }
}

// ---------------------------------------------------------------------------
// z = B r (block-diagonal inverse), one thread per block row (the block's r
// in registers, the inverse read coalesced across the warp's 32 block rows,
// loads beyond the block's own size predicated off), with the dot products
// the following step needs.
//   MODE 0 (setup):  (z, z)                  -> rnorm0, ttol, rho = (r0, r0)
//   MODE 1 (v):      (z, a)                  -> alpha = rho / (v, r0)
//   MODE 2 (t):      (a, z) (z, z) (a, a)    -> omega = (s,t) / (t,t)
// ---------------------------------------------------------------------------
constexpr int kApplyThreads = 128;

// Owned block rows of one slab in a z-slab decomposition: [b0, b1) in the
// matrix continuum, [b2, b3) in the fracture continuum (local numbering).
struct Owned {
    long b0 = 0, b1 = 0, b2 = 0, b3 = 0;
    __device__ __forceinline__ bool block(long b) const { return (b >= b0 && b < b1) || (b >= b2 && b < b3); }
};

// DIST: the distributed form (one slab): the dot products are summed over
// the owned block rows only and written to dots[] for the host to sum over
// the slabs; the scalar step is left to dksp_scalar_kernel.
// TR: apply the transposed inverse blocks (the preconditioner of a solve
// with the transposed matrix).
template <int N, int MODE, bool DIST = false, bool TR = false>
__global__ void __launch_bounds__(kApplyThreads) bjac_apply_kernel(const KView v, const double *__restrict__ inv,
                                                                    const double *__restrict__ r,
                                                                    double *__restrict__ z,
                                                                    const double *__restrict__ a, double *part,
                                                                    KspScal *s, Owned own = Owned(),
                                                                    double *dots = nullptr) {
    if (s->reason != kItersRunning) return;
    constexpr int BS = 2 * N + 4;
    const long nb = 2 * v.n;
    double acc[kParts] = {0, 0, 0};
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long)gridDim.x * blockDim.x) {
        const long off = v.rowoff[b];
        const int bs = (int)(v.rowoff[b + 1] - off);
        const double *ib = inv + ((b >> 5) * (BS * BS)) * 32 + (b & 31);
        double rv[BS], zv[BS];
#pragma unroll
        for (int j = 0; j < BS; j++) {
            rv[j] = j < bs ? __ldg(r + off + j) : 0.0;
            zv[j] = 0;
        }
#pragma unroll
        for (int j = 0; j < BS; j++) {
            if (j >= bs) break;
#pragma unroll
            for (int i = 0; i < BS; i++)
                if (i < bs) zv[i] += __ldg(ib + 32 * (TR ? (i * BS + j) : (j * BS + i))) * rv[j];
        }
        const bool count = !DIST || own.block(b);
#pragma unroll
        for (int i = 0; i < BS; i++) {
            if (i >= bs) break;
            const double t = zv[i];
            z[off + i] = t;
            if (!count) continue;
            if (MODE == 0) {
                acc[0] += t * t;
            } else if (MODE == 1) {
                acc[0] += t * a[off + i];
            } else {
                const double sv = a[off + i];
                acc[0] += sv * t;
                acc[1] += t * t;
                acc[2] += sv * sv;
            }
        }
    }
    double tot[kParts];
    if (!publish_partials<kParts>(acc, part, s, tot)) return;
    if (DIST) {
#pragma unroll
        for (int q = 0; q < kParts; q++) dots[q] = tot[q];
        return;
    }
    if (MODE == 0) {
        // set-up of KSPSolve_BCGS: |r_0| and the convergence test at iteration 0
        const double rn = sqrt(tot[0]);
        s->rnorm0 = rn;
        s->rnorm = rn;
        s->ttol = fmax(s->rtol * rn, s->atol);
        s->its = 0;
        converged_test(s, rn);
        s->rho = tot[0];   // (r, r0) with r0 = r
        s->rhoold = 1.0;
        s->alpha = 1.0;
        s->omegaold = 1.0;
        s->beta = (s->rho / s->rhoold) * (s->alpha / s->omegaold);
    } else if (MODE == 1) {
        const double d1 = tot[0];
        if (!isfinite(d1)) s->reason = kDivergedNanOrInf;
        else if (d1 == 0.0) s->reason = kDivergedBreakdown;
        else s->alpha = s->rho / d1;
    } else {
        const double d1 = tot[0], d2 = tot[1], ss = tot[2];
        if (d2 == 0.0) {
            // t = 0: if s = 0 too, x + alpha p solves the system
            if (ss != 0.0) {
                s->reason = kDivergedBreakdown;
            } else {
                s->omega = 0.0;
                s->its += 1;
                s->rnorm = 0.0;
                s->reason = kFinishWithP;
            }
        } else {
            s->omega = d1 / d2;
        }
    }
}

// p <- r + beta (p - omega_old v)
__global__ void __launch_bounds__(256) bcgs_p_kernel(long n, const double *__restrict__ r, double *__restrict__ p,
                                                     const double *__restrict__ v, const KspScal *s) {
    if (s->reason != kItersRunning) return;
    const double beta = s->beta, ob = s->omegaold * s->beta;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = r[i] + beta * p[i] - ob * v[i];
}

// s <- r - alpha v
__global__ void __launch_bounds__(256) bcgs_s_kernel(long n, const double *__restrict__ r,
                                                     const double *__restrict__ v, double *__restrict__ sv,
                                                     const KspScal *s) {
    if (s->reason != kItersRunning) return;
    const double alpha = s->alpha;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        sv[i] = r[i] - alpha * v[i];
}

// x += alpha p + omega s; r <- s - omega t; |r|^2 and (r, r0) -> the
// convergence test and the next iteration's rho and beta.
__global__ void __launch_bounds__(kRedThreads) bcgs_xr_kernel(long n, double *__restrict__ x,
                                                               const double *__restrict__ p,
                                                               const double *__restrict__ sv,
                                                               const double *__restrict__ t,
                                                               double *__restrict__ r,
                                                               const double *__restrict__ r0, double *part,
                                                               KspScal *s) {
    const int reason = s->reason;
    if (reason != kItersRunning && reason != kFinishWithP) return;
    const double alpha = s->alpha, omega = s->omega;
    double acc[2] = {0, 0};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (reason == kFinishWithP) {
            x[i] += alpha * p[i];
            continue;
        }
        const double si = sv[i];
        x[i] += alpha * p[i] + omega * si;
        const double ri = si - omega * t[i];
        r[i] = ri;
        acc[0] += ri * ri;
        acc[1] += ri * r0[i];
    }
    double tot[2];
    if (!publish_partials<2>(acc, part, s, tot)) return;
    if (reason == kFinishWithP) {
        s->reason = kConvergedRtol;
        return;
    }
    const double dp = sqrt(tot[0]);
    const double rho = s->rho;
    s->rhoold = rho;
    s->omegaold = omega;
    s->its += 1;
    s->rnorm = dp;
    converged_test(s, dp);
    if (s->reason == kItersRunning && rho == 0.0) s->reason = kDivergedBreakdown;
    if (s->reason == kItersRunning && s->its >= s->max_it) s->reason = kDivergedIts;
    s->rho = tot[1];
    s->beta = (s->rho / s->rhoold) * (s->alpha / s->omegaold);
}

// r0 <- r, p <- 0, v <- 0, x <- 0
__global__ void __launch_bounds__(256) bcgs_setup_kernel(long n, const double *__restrict__ r, double *__restrict__ r0,
                                                         double *__restrict__ p, double *__restrict__ v,
                                                         double *__restrict__ x) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        r0[i] = r[i];
        p[i] = 0;
        v[i] = 0;
        x[i] = 0;
    }
}

// ---------------------------------------------------------------------------
// Distributed form: one slab of a z-slab decomposition runs the iteration
// above split at its dot products (PETSc runs KSPBCGS the same way over MPI
// ranks, with VecDot / VecNorm reductions across the ranks).  Each stage's
// dot products are summed over the slab's owned rows into dots[]; the host
// sums dots[] over the slabs (an all-reduce, stream-ordered) and the next
// stage's dksp_scalar_kernel takes the scalar step from the sums.  Vector
// updates run over every local row; the host refills the ghost rows of p and
// s from the neighbouring slabs before each product.  Stages of one
// iteration:
//   1  p <- r + beta (p - omega_old v)                     [ghost rows of p]
//   2  t <- A p, v <- B t, dots = (v, r0)                  [sum]
//   3  alpha; s <- r - alpha v                             [ghost rows of s]
//   4  w <- A s, t <- B w, dots = (s, t) (t, t) (s, s)     [sum]
//   5  omega; x += alpha p + omega s, r <- s - omega t, dots = |r|^2 (r, r0)
//                                                          [sum]
//   6  convergence test, rho, beta
// The set-up (r <- B b, dots = |r|^2 [sum]) is followed by stage 0, the
// set-up's scalar step.  Every slab takes the same scalar steps from the
// same sums, so all slabs stop at the same iteration.
// ---------------------------------------------------------------------------

// x += alpha p + omega s; r <- s - omega t; |r|^2 and (r, r0) over the owned
// rows ([rowoff[b0], rowoff[b1]) and [rowoff[b2], rowoff[b3])) into dots.
__global__ void __launch_bounds__(kRedThreads) dbcgs_xr_kernel(long n, double *__restrict__ x,
                                                                const double *__restrict__ p,
                                                                const double *__restrict__ sv,
                                                                const double *__restrict__ t,
                                                                double *__restrict__ r,
                                                                const double *__restrict__ r0,
                                                                const long *__restrict__ rowoff, Owned own,
                                                                double *part, double *dots, KspScal *s) {
    const int reason = s->reason;
    if (reason != kItersRunning && reason != kFinishWithP) return;
    const long m0 = rowoff[own.b0], m1 = rowoff[own.b1], f0 = rowoff[own.b2], f1 = rowoff[own.b3];
    const double alpha = s->alpha, omega = s->omega;
    double acc[2] = {0, 0};
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (reason == kFinishWithP) {
            x[i] += alpha * p[i];
            continue;
        }
        const double si = sv[i];
        x[i] += alpha * p[i] + omega * si;
        const double ri = si - omega * t[i];
        r[i] = ri;
        if ((i >= m0 && i < m1) || (i >= f0 && i < f1)) {
            acc[0] += ri * ri;
            acc[1] += ri * r0[i];
        }
    }
    double tot[2];
    if (!publish_partials<2>(acc, part, s, tot)) return;
    dots[0] = tot[0];
    dots[1] = tot[1];
}

// The scalar step of a stage from the summed dot products (the tails of
// bjac_apply_kernel MODE 0 / 1 / 2 and bcgs_xr_kernel above).
__global__ void dksp_scalar_kernel(KspScal *s, const double *dots, int stage) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (stage == 0) {
        const double rn = sqrt(dots[0]);
        s->rnorm0 = rn;
        s->rnorm = rn;
        s->ttol = fmax(s->rtol * rn, s->atol);
        s->its = 0;
        converged_test(s, rn);
        s->rho = dots[0];
        s->rhoold = 1.0;
        s->alpha = 1.0;
        s->omegaold = 1.0;
        s->beta = (s->rho / s->rhoold) * (s->alpha / s->omegaold);
    } else if (stage == 3) {
        if (s->reason != kItersRunning) return;
        const double d1 = dots[0];
        if (!isfinite(d1)) s->reason = kDivergedNanOrInf;
        else if (d1 == 0.0) s->reason = kDivergedBreakdown;
        else s->alpha = s->rho / d1;
    } else if (stage == 5) {
        if (s->reason != kItersRunning) return;
        const double d1 = dots[0], d2 = dots[1], ss = dots[2];
        if (d2 == 0.0) {
            if (ss != 0.0) {
                s->reason = kDivergedBreakdown;
            } else {
                s->omega = 0.0;
                s->its += 1;
                s->rnorm = 0.0;
                s->reason = kFinishWithP;
            }
        } else {
            s->omega = d1 / d2;
        }
    } else if (stage == 6) {
        if (s->reason == kFinishWithP) {
            s->reason = kConvergedRtol;
            return;
        }
        if (s->reason != kItersRunning) return;
        const double dp = sqrt(dots[0]);
        const double rho = s->rho, omega = s->omega;
        s->rhoold = rho;
        s->omegaold = omega;
        s->its += 1;
        s->rnorm = dp;
        converged_test(s, dp);
        if (s->reason == kItersRunning && rho == 0.0) s->reason = kDivergedBreakdown;
        if (s->reason == kItersRunning && s->its >= s->max_it) s->reason = kDivergedIts;
        s->rho = dots[1];
        s->beta = (s->rho / s->rhoold) * (s->alpha / s->omegaold);
    }
}

}  // namespace osrk
