// Adjoint of the flash: sensitivities of a converged flash result to the
// binary-interaction coefficients, the feed and the pressure.
//
// A two-phase cell's result u = (x, y, L) solves
//   G_i = ln x_i + ln phi_i^L(x) - ln y_i - ln phi_i^V(y) = 0   (equal fugacity)
//   H_i = z_i - L x_i - (1 - L) y_i = 0                        (material balance)
//   S   = sum_i (x_i - y_i) = 0                                (Rachford-Rice)
// to the reference's stopping tolerances (SuccFalsh,
// compsim/Init_Calcs.cpp:571-738).  By the implicit-function theorem a
// cotangent (xbar, ybar, Lbar) on u gives theta_bar = -lambda^T dF/dtheta with
// J^T lambda = (xbar, ybar, Lbar), J = dF/du, F = (G, H, S).  The 2N+1
// system reduces exactly to N+1 unknowns: with A_x = D_x + Phi_x^T (D_x =
// diag(1/x), Phi_x[i][k] = d ln phi_i^L/d x_k) and A_y likewise,
//   [ (1-L) A_x + L A_y      1 ] [lambda_G]   [ (1-L) xbar - L ybar        ]
//   [ d^T (A_x - A_y)        0 ] [lambda_S] = [ Lbar + d^T (xbar + ybar)   ]
// with d = y - x, and lambda_H = (A_x - A_y) lambda_G - xbar - ybar.  Then
//   kij_bar = -sum_i lambda_G,i (d ln phi_i^L/d k - d ln phi_i^V/d k),
//   z_bar = -lambda_H,   P_bar = -sum_i lambda_G,i (d ln phi_i^L/dP - d ln phi_i^V/dP).
// The reference has no adjoint; the derivative blocks Phi are the flash's
// own (the fugacity rows of IteratorJacobian,
// compsim/Petsc_Functions.cpp:30243-30372).  One-phase cells: the present
// phase is the feed (its cotangent goes to z_bar) and nothing depends on
// k_ij; the incipient phase's composition is the reference's unconverged
// two-step estimate and carries no sensitivity here.
#pragma once
#include "flash_kernels.cuh"

namespace osr {

// sum_i wt_i d ln(phi_i)/d k_pq of one phase, subtracted into kb[p N + q]:
// k_pq enters as sqrt(a_p a_q)(1 - k_pq) in the mixing sum C_a and in row p
// of s_i = sqrt(a_i) sum_j (1 - k_ij) w_j sqrt(a_j); Z follows A through the
// cubic (dZ/dA = -(Z - B)/f'(Z)).
template <int N>
__device__ __forceinline__ void lnphi_kij_vjp(const FluidTable<N> &f, const double *sa, double P, double T,
                                              const double *w, double Z, const double *wt, double *kb) {
    double u[N], v[N];
#pragma unroll
    for (int i = 0; i < N; i++) u[i] = w[i] * sa[i];
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
    const bool srk = f.srk != 0;
    const double rt = kR * T;
    const double pa = P / (rt * rt), A = Ca * pa, B = Cb * (P / rt);
    const double U = srk ? B : 2 * B, W = srk ? 0.0 : B;
    const double d1 = srk ? 1.0 : 1 + kSqrt2, d2 = srk ? 0.0 : 1 - kSqrt2;
    const double fp = 3 * Z * Z - 2 * Z * (1 + B - U) + A - B * U - U - W * W;
    const double dZdA = -(Z - B) / fp;
    const double DD = A / (B * (d1 - d2)), FF = log((Z + d2 * B) / (Z + d1 * B));
    const double dFF = 1 / (Z + d2 * B) - 1 / (Z + d1 * B);
    double gZ = 0, gDD = 0, gCa = 0, gs[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        const double si = sa[i] * v[i];
        const double t1 = f.b[i] / Cb, EE = 2 * si / Ca - t1;
        gZ += wt[i] * (t1 - 1 / (Z - B) + DD * EE * dFF);
        gDD += wt[i] * FF * EE;
        gCa -= wt[i] * DD * FF * 2 * si / (Ca * Ca);
        gs[i] = wt[i] * DD * FF * 2 / Ca;
    }
    gCa += gZ * dZdA * pa + gDD * DD / Ca;
#pragma unroll
    for (int p = 0; p < N; p++)
#pragma unroll
        for (int q = 0; q < N; q++) kb[p * N + q] -= sa[p] * sa[q] * w[q] * (gCa * w[p] + gs[p]);
}

// Dense (N+1) x (N+1) solve, partial pivoting, row-major in local memory;
// false when a pivot is exactly zero.
template <int M>
__device__ bool solve_small(double *A, double *b) {
#pragma unroll 1
    for (int k = 0; k < M; k++) {
        int p = k;
        for (int i = k + 1; i < M; i++)
            if (fabs(A[i * M + k]) > fabs(A[p * M + k])) p = i;
        if (A[p * M + k] == 0) return false;
        if (p != k) {
            for (int j = 0; j < M; j++) {
                const double t = A[k * M + j];
                A[k * M + j] = A[p * M + j];
                A[p * M + j] = t;
            }
            const double t = b[k];
            b[k] = b[p];
            b[p] = t;
        }
        const double r = 1 / A[k * M + k];
        for (int i = k + 1; i < M; i++) {
            const double l = A[i * M + k] * r;
            for (int j = k; j < M; j++) A[i * M + j] -= l * A[k * M + j];
            b[i] -= l * b[k];
        }
    }
#pragma unroll 1
    for (int i = M - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < M; j++) s -= A[i * M + j] * b[j];
        b[i] = s / A[i * M + i];
    }
    return true;
}

struct AdjointIO {
    const double *P, *T, *z;
    long n;
    const signed char *label;
    const double *L, *x, *y, *Zl, *Zg;
    const double *xbar, *ybar, *Lbar;
    double *z_bar, *P_bar;   // optional
    double *partials;        // [gridDim.x][N*N] per-block sums of kij_bar
    unsigned *singular;      // count of two-phase cells with a singular system
};

template <int N>
struct AdjointArgs {
    FluidTable<N> f;
    AdjointIO io;
};

constexpr int kAdjThreads = 128;

// One thread per cell (grid-stride, fixed grid: every thread's cells and
// their order are fixed, so the kij sums are deterministic).  Each thread
// accumulates its cells' kij_bar, the warp and the block reduce it in fixed
// order, and the block writes its partial sum.
template <int N>
__global__ void __launch_bounds__(kAdjThreads) flash_adjoint_kernel(const __grid_constant__ AdjointArgs<N> a) {
    constexpr int M = N + 1;
    const AdjointIO &io = a.io;
    const FluidTable<N> &f = a.f;
    double kb[N * N];
#pragma unroll
    for (int e = 0; e < N * N; e++) kb[e] = 0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < io.n; c += stride) {
        const signed char lab = io.label[c];
        double pbar = 0;
        if (lab != 0) {
            // one phase: the present phase is the feed
            if (io.z_bar)
#pragma unroll
                for (int i = 0; i < N; i++)
                    io.z_bar[(long)i * io.n + c] = lab > 0 ? io.xbar[(long)i * io.n + c] : io.ybar[(long)i * io.n + c];
            if (io.P_bar) io.P_bar[c] = 0;
            continue;
        }
        const double P = io.P[c], T = io.T[c], L = io.L[c];
        double sa[N], xs[N], ys[N], xb[N], yb[N], d[N];
        bool live[N];
        sqrt_a<N>(f, T, sa);
#pragma unroll
        for (int i = 0; i < N; i++) {
            xs[i] = io.x[(long)i * io.n + c];
            ys[i] = io.y[(long)i * io.n + c];
            xb[i] = io.xbar[(long)i * io.n + c];
            yb[i] = io.ybar[(long)i * io.n + c];
            d[i] = ys[i] - xs[i];
            live[i] = xs[i] > 0 && ys[i] > 0;
        }
        double dxl[N * N], dxg[N * N], dpl[N], dpg[N];
        phase_derivs_into<N>(
            f, sa, P, T, xs, io.Zl[c], [&](int i, int k, double v) { dxl[i * N + k] = v; },
            [&](int i, double v) { dpl[i] = v; });
        phase_derivs_into<N>(
            f, sa, P, T, ys, io.Zg[c], [&](int i, int k, double v) { dxg[i * N + k] = v; },
            [&](int i, double v) { dpg[i] = v; });
        double Ms[M * M], r[M];
        double rN = io.Lbar[c];
#pragma unroll 1
        for (int k = 0; k < N; k++) {
            double ck = 0;
            for (int i = 0; i < N; i++) {
                const double Ax = (i == k && live[i] ? 1 / xs[i] : 0.0) + dxl[k * N + i];
                const double Ay = (i == k && live[i] ? 1 / ys[i] : 0.0) + dxg[k * N + i];
                Ms[i * M + k] = (live[i] && live[k]) ? (1 - L) * Ax + L * Ay : (i == k ? 1.0 : 0.0);
                ck += live[i] ? d[i] * (Ax - Ay) : 0.0;
            }
            Ms[k * M + N] = live[k] ? 1.0 : 0.0;
            Ms[N * M + k] = live[k] ? ck : 0.0;
            r[k] = live[k] ? (1 - L) * xb[k] - L * yb[k] : 0.0;
            rN += live[k] ? d[k] * (xb[k] + yb[k]) : 0.0;
        }
        Ms[N * M + N] = 0;
        r[N] = rN;
        if (!solve_small<M>(Ms, r)) {
            atomicAdd(io.singular, 1u);
            if (io.z_bar)
                for (int i = 0; i < N; i++) io.z_bar[(long)i * io.n + c] = 0;
            if (io.P_bar) io.P_bar[c] = 0;
            continue;
        }
        double wl[N], wg[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            const double lg = live[i] ? r[i] : 0.0;
            wl[i] = -lg;
            wg[i] = lg;
            pbar -= lg * (dpl[i] - dpg[i]);
        }
        if (io.z_bar) {
#pragma unroll 1
            for (int i = 0; i < N; i++) {
                double lh = 0;
                if (live[i]) {
                    lh = -xb[i] - yb[i] + r[i] / xs[i] - r[i] / ys[i];
                    for (int k = 0; k < N; k++)
                        if (live[k]) lh += (dxl[k * N + i] - dxg[k * N + i]) * r[k];
                }
                io.z_bar[(long)i * io.n + c] = -lh;
            }
        }
        if (io.P_bar) io.P_bar[c] = pbar;
        lnphi_kij_vjp<N>(f, sa, P, T, xs, io.Zl[c], wl, kb);
        lnphi_kij_vjp<N>(f, sa, P, T, ys, io.Zg[c], wg, kb);
    }
    // kij_bar: warp sums by shuffles, then the block's warps in order
    __shared__ double part[kAdjThreads / 32][N * N];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int e = 0; e < N * N; e++) {
        double v = kb[e];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) part[warp][e] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        double s = 0;
        for (int w = 0; w < kAdjThreads / 32; w++) s += part[w][e];
        io.partials[(long)blockIdx.x * N * N + e] = s;
    }
}

// kij_bar[e] = the blocks' partials summed in block order.
__global__ void adjoint_reduce_kernel(const double *partials, int blocks, int entries, double *kij_bar) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= entries) return;
    double s = 0;
    for (int b = 0; b < blocks; b++) s += partials[(long)b * entries + e];
    kij_bar[e] = s;
}

}  // namespace osr
