// Host side of the device linear solve (ksp_kernels.cuh): the KSPSolve of
// SolveNonLinear (compsim/PetscAUX.cpp:631-646, 672-698) on the compact
// Jacobian, and the matrix-vector product alone (MatMult).
#include <cuda_runtime.h>
#include <cstddef>
#include <cstring>
#include <functional>
#include <vector>
#include "grid_internal.h"
#include "ksp_kernels.cuh"

struct osr_ksp_work {
    long rows_cap = 0, blocks = 0;
    int nc = 0;
    double *r = nullptr, *r0 = nullptr, *p = nullptr, *v = nullptr, *t = nullptr, *s = nullptr, *w = nullptr;
    double *inv = nullptr;
    double *part = nullptr;
    osrk::KspScal *scal = nullptr;   // device
    osrk::KspScal *host = nullptr;   // pinned
    // one batch of iterations captured as a CUDA graph, replayed while the
    // matrix values, solution vector, row count and batch size stay the same
    cudaStream_t cap = nullptr;
    cudaGraphExec_t batch = nullptr;
    const double *g_vals = nullptr;
    double *g_x = nullptr;
    long g_rows = -1;
    int g_every = 0;
    // the whole solve as one graph: the scalars in, block-Jacobi set-up, a
    // device-side while loop over batches of iterations, the scalars out
    cudaGraphExec_t whole = nullptr;
    const double *w_vals = nullptr, *w_b = nullptr;
    double *w_x = nullptr;
    long w_rows = -1;
    int w_every = 0, w_max = 0;
    bool whole_failed = false;
};

// One slab's part of a distributed solve (osr_dksp_*): its scalars and the
// caller's vectors; the other vectors, the block inverses and the partial
// sums are the grid's solve workspace.
struct osr_dksp {
    osr_grid *g = nullptr;
    osrk::KspScal *scal = nullptr;   // device
    osrk::KspScal *host = nullptr;   // pinned
    const double *vals = nullptr, *b = nullptr;
    double *x = nullptr, *p = nullptr, *s = nullptr, *dots = nullptr;
    osrk::Owned own;
    long rows = 0;
};

namespace osr {

#define KSP_CUDA(call)                                     \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return OSR_ERR_CUDA;        \
    } while (0)

void ksp_free(osr_grid &g) {
    osr_ksp_work *k = g.ksp;
    if (!k) return;
    void *ptrs[] = {k->r, k->r0, k->p, k->v, k->t, k->s, k->w, k->inv, k->part, k->scal};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (k->host) cudaFreeHost(k->host);
    if (k->batch) cudaGraphExecDestroy(k->batch);
    if (k->cap) cudaStreamDestroy(k->cap);
    delete k;
    g.ksp = nullptr;
}

// Vectors sized for the largest row layout (every cell-medium two-phase), so
// phase changes never reallocate.
static osr_status ksp_ensure(osr_grid &g) {
    if (g.ksp) return OSR_OK;
    osr_ksp_work *k = new osr_ksp_work();
    g.ksp = k;
    const int bs = 2 * g.nc + 4;
    k->nc = g.nc;
    k->blocks = 2 * g.cells;
    k->rows_cap = k->blocks * bs;
    const size_t vb = (size_t)k->rows_cap * sizeof(double);
    double **vecs[] = {&k->r, &k->r0, &k->p, &k->v, &k->t, &k->s, &k->w};
    for (double **q : vecs) KSP_CUDA(cudaMalloc((void **)q, vb));
    KSP_CUDA(cudaMalloc((void **)&k->inv, (size_t)((k->blocks + 31) / 32) * 32 * bs * bs * sizeof(double)));
    KSP_CUDA(cudaMalloc((void **)&k->part, (size_t)osrk::kParts * osrk::kMaxRedBlocks * sizeof(double)));
    KSP_CUDA(cudaMalloc((void **)&k->scal, sizeof(osrk::KspScal)));
    KSP_CUDA(cudaMallocHost((void **)&k->host, sizeof(osrk::KspScal)));
    return OSR_OK;
}

static osrk::KView kview(const osr_grid &g, const double *vals) {
    osrk::KView v;
    v.nc = g.nc;
    v.nx = g.nx;
    v.ny = g.ny;
    v.nz = g.nz;
    v.n = g.cells;
    v.rows = g.n_rows;
    v.rowoff = g.rowoff;
    v.lab_m = g.m[0].label;
    v.lab_f = g.m[1].label;
    v.vals = vals;
    v.entries = osrj::Layout(g.nc).ET;
    return v;
}

static unsigned spmv_blocks(long nb, int lanes) {
    const long per_cta = (32 / lanes) * (osrk::kSpmvThreads / 32);   // block rows per CTA and sweep
    long b = (nb + per_cta - 1) / per_cta;
    if (b > 148L * 64) b = 148L * 64;
    return (unsigned)(b < 1 ? 1 : b);
}

static unsigned vec_blocks(long n) {
    long b = (n + 255) / 256;
    if (b > 148L * 16) b = 148L * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

// CTAs of the reducing kernels: enough to cover the work in one sweep, at
// most kMaxRedBlocks (the partial-sum buffer).
static unsigned red_blocks(long work, int per_cta) {
    long b = (work + per_cta - 1) / per_cta;
    if (b > osrk::kMaxRedBlocks) b = osrk::kMaxRedBlocks;
    return (unsigned)(b < 1 ? 1 : b);
}

static unsigned inv_blocks(long nb) {
    long b = (nb + osrk::kInvWarps - 1) / osrk::kInvWarps;
    if (b > 148L * 64) b = 148L * 64;
    return (unsigned)(b < 1 ? 1 : b);
}

// y = A x: two lanes per block row on large grids (128-byte runs per
// slot), four below osrk::kSpmvRowForm block rows (shorter dependent chains
// where the grid alone cannot fill the GPU).
template <int N>
static void spmv_launch(const osrk::KView &v, const double *x, double *y, const osrk::KspScal *sc,
                        cudaStream_t st) {
    const long nb = 2 * v.n;
    if (nb >= osrk::kSpmvRowForm)
        osrk::spmv_kernel<N, 2><<<spmv_blocks(nb, 2), osrk::kSpmvThreads, 0, st>>>(v, x, y, sc);
    else
        osrk::spmv_kernel<N, 4><<<spmv_blocks(nb, 4), osrk::kSpmvThreads, 0, st>>>(v, x, y, sc);
}

template <int N>
static osr_status spmv_n(const osr_grid &g, const double *vals, const double *x, double *y, cudaStream_t st) {
    const osrk::KView v = kview(g, vals);
    spmv_launch<N>(v, x, y, nullptr, st);
    KSP_CUDA(cudaGetLastError());
    return OSR_OK;
}

// Condition of the solve graph's while loop: another batch while the solve
// is running, at most max_batches in all (KspScal.pad counts the batches; it
// is zero when the scalars are copied in).  The bound holds whatever the
// scalars say, so the loop always ends.
__global__ void bcgs_continue_kernel(cudaGraphConditionalHandle h, osrk::KspScal *s, int max_batches) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int done = ++s->pad;
        const bool go = s->reason == osrk::kItersRunning && done < max_batches;
        cudaGraphSetConditional(h, go ? 1u : 0u);
    }
}

// Launch shapes and operands of one system.
template <int N>
struct SolvePlan {
    osrk::KView v;
    long n, nb;
    unsigned vbk, ib, tpb, atb, ab, xb;
    const double *b;
    double *x;
};

template <int N>
static SolvePlan<N> solve_plan(const osr_grid &g, const double *vals, const double *b, double *x) {
    SolvePlan<N> p;
    p.v = kview(g, vals);
    p.n = g.n_rows;
    p.nb = 2 * g.cells;
    p.vbk = vec_blocks(p.n);
    p.ib = inv_blocks(p.nb);
    p.tpb = 32 * osrk::kInvWarps;
    p.atb = osrk::kApplyThreads;
    p.ab = red_blocks(p.nb, osrk::kApplyThreads);
    p.xb = red_blocks(p.n, 4 * osrk::kRedThreads);
    p.b = b;
    p.x = x;
    return p;
}

// scalars in (from the pinned host copy), block-Jacobi inverse, r = B b,
// the BiCGStab set-up
template <int N>
static void solve_prologue(osr_ksp_work &k, const SolvePlan<N> &p, cudaStream_t st) {
    cudaMemcpyAsync(k.scal, k.host, sizeof(osrk::KspScal), cudaMemcpyHostToDevice, st);
    osrk::bjac_invert_kernel<N><<<p.ib, p.tpb, 0, st>>>(p.v, k.inv, k.scal);
    osrk::bjac_apply_kernel<N, 0><<<p.ab, p.atb, 0, st>>>(p.v, k.inv, p.b, k.r, nullptr, k.part, k.scal);
    osrk::bcgs_setup_kernel<<<p.vbk, 256, 0, st>>>(p.n, k.r, k.r0, k.p, k.v, p.x);
}

template <int N>
static void solve_iterations(osr_ksp_work &k, const SolvePlan<N> &p, cudaStream_t st, int count) {
    for (int q = 0; q < count; q++) {
        osrk::bcgs_p_kernel<<<p.vbk, 256, 0, st>>>(p.n, k.r, k.p, k.v, k.scal);
        spmv_launch<N>(p.v, k.p, k.t, k.scal, st);
        osrk::bjac_apply_kernel<N, 1><<<p.ab, p.atb, 0, st>>>(p.v, k.inv, k.t, k.v, k.r0, k.part, k.scal);
        osrk::bcgs_s_kernel<<<p.vbk, 256, 0, st>>>(p.n, k.r, k.v, k.s, k.scal);
        spmv_launch<N>(p.v, k.s, k.w, k.scal, st);
        osrk::bjac_apply_kernel<N, 2><<<p.ab, p.atb, 0, st>>>(p.v, k.inv, k.w, k.t, k.s, k.part, k.scal);
        osrk::bcgs_xr_kernel<<<p.xb, osrk::kRedThreads, 0, st>>>(p.n, p.x, k.p, k.s, k.t, k.r, k.r0, k.part,
                                                                  k.scal);
    }
}

// The whole solve as one graph: `pre` (work captured ahead of it, or null),
// the prologue, a while node whose body is one batch of `every` iterations
// and the continue test (at most max_it / every batches), the scalars back
// to the pinned host copy, then `post` (or null).  False when any part of
// the capture fails (nothing is left instantiated).
template <int N>
static bool build_solve_graph(osr_ksp_work &k, const SolvePlan<N> &p, int every, int max_it,
                              const std::function<void(cudaStream_t)> *pre,
                              const std::function<void(cudaStream_t)> *post, const GraphExtend *extend,
                              cudaGraphExec_t *out) {
    *out = nullptr;
    if (!k.cap && cudaStreamCreateWithFlags(&k.cap, cudaStreamNonBlocking) != cudaSuccess) return false;
    const cudaStreamCaptureMode mode = pre || post ? cudaStreamCaptureModeRelaxed : cudaStreamCaptureModeThreadLocal;
    cudaGraph_t G = nullptr;
    bool ok = cudaGraphCreate(&G, 0) == cudaSuccess;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraphNode_t wnode = nullptr;
    cudaGraphConditionalHandle handle;
    if (ok) ok = cudaGraphConditionalHandleCreate(&handle, G, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) ok = cudaStreamBeginCaptureToGraph(k.cap, G, nullptr, nullptr, 0, mode) == cudaSuccess;
    if (ok) {
        if (pre) (*pre)(k.cap);
        solve_prologue<N>(k, p, k.cap);
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        ok = cudaStreamGetCaptureInfo(k.cap, &cs, nullptr, &cg, &deps, &ndeps) == cudaSuccess &&
             cs == cudaStreamCaptureStatusActive;
        std::vector<cudaGraphNode_t> tail(deps, deps + (ok ? ndeps : 0));
        cudaGraph_t og = nullptr;
        ok = (cudaStreamEndCapture(k.cap, &og) == cudaSuccess) && ok;
        if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&wnode, G, tail.data(), tail.size(), &cp) == cudaSuccess;
            cudaGraph_t body = ok ? cp.conditional.phGraph_out[0] : nullptr;
            if (ok) ok = cudaStreamBeginCaptureToGraph(k.cap, body, nullptr, nullptr, 0, mode) == cudaSuccess;
            if (ok) {
                solve_iterations<N>(k, p, k.cap, every);
                bcgs_continue_kernel<<<1, 32, 0, k.cap>>>(handle, k.scal, max_it / every);
                cudaGraph_t bout = nullptr;
                ok = cudaStreamEndCapture(k.cap, &bout) == cudaSuccess;
                size_t body_nodes = 0;
                // the body must hold the continue test (else the loop could not end)
                if (ok) ok = cudaGraphGetNodes(body, nullptr, &body_nodes) == cudaSuccess &&
                             body_nodes == (size_t)(7 * every + 1);
            }
            if (ok) ok = cudaStreamBeginCaptureToGraph(k.cap, G, &wnode, nullptr, 1, mode) == cudaSuccess;
            if (ok) {
                cudaMemcpyAsync(k.host, k.scal, sizeof(osrk::KspScal), cudaMemcpyDeviceToHost, k.cap);
                if (post) (*post)(k.cap);
                std::vector<cudaGraphNode_t> leaves;
                if (extend) {
                    cudaStreamCaptureStatus cs2;
                    const cudaGraphNode_t *d2 = nullptr;
                    size_t n2 = 0;
                    ok = cudaStreamGetCaptureInfo(k.cap, &cs2, nullptr, nullptr, &d2, &n2) == cudaSuccess &&
                         cs2 == cudaStreamCaptureStatusActive;
                    if (ok) leaves.assign(d2, d2 + n2);
                }
                cudaGraph_t eout = nullptr;
                ok = (cudaStreamEndCapture(k.cap, &eout) == cudaSuccess) && ok;
                if (ok && extend) ok = (*extend)(G, k.cap, leaves);
            }
        }
    }
    if (ok) ok = cudaGraphInstantiate(out, G, 0) == cudaSuccess;
    if (!ok) *out = nullptr;
    if (G) cudaGraphDestroy(G);
    cudaGetLastError();
    return ok;
}

static void ksp_set_host(osr_ksp_work &k, const osr_ksp_opts &o) {
    osrk::KspScal h;
    std::memset(&h, 0, sizeof(h));
    h.rtol = o.rtol;
    h.atol = o.atol;
    h.dtol = o.dtol;
    h.max_it = o.max_it;
    *k.host = h;
}

static void ksp_read_host(const osr_ksp_work &k, osr_ksp_info *info) {
    if (!info) return;
    info->reason = k.host->reason == osrk::kItersRunning ? osrk::kDivergedIts : k.host->reason;
    info->its = k.host->its;
    info->rnorm0 = k.host->rnorm0;
    info->rnorm = k.host->rnorm;
}

template <int N>
static osr_status solve_n(osr_grid &g, const double *vals, const double *b, double *x, const osr_ksp_opts &o,
                          osr_ksp_info *info, cudaStream_t st) {
    osr_status rc = ksp_ensure(g);
    if (rc != OSR_OK) return rc;
    osr_ksp_work &k = *g.ksp;
    const SolvePlan<N> p = solve_plan<N>(g, vals, b, x);
    const long n = p.n;
    ksp_set_host(k, o);
    const int every = o.check_every > 0 ? o.check_every : 8;
    // The whole solve as one graph: one launch and one synchronisation per
    // solve.  Used when the iteration cap is a whole number of batches (so
    // the graph stops exactly where the host loop would); kept while the
    // system's buffers and size stay the same.
    if (k.whole && (k.w_vals != vals || k.w_b != b || k.w_x != x || k.w_rows != n || k.w_every != every ||
                    k.w_max != o.max_it)) {
        cudaGraphExecDestroy(k.whole);
        k.whole = nullptr;
    }
    if (!k.whole && !k.whole_failed && o.max_it >= every && o.max_it % every == 0) {
        if (!build_solve_graph<N>(k, p, every, o.max_it, nullptr, nullptr, nullptr, &k.whole))
            k.whole_failed = true;   // the host-driven batches below serve every later solve
        if (k.whole) {
            k.w_vals = vals;
            k.w_b = b;
            k.w_x = x;
            k.w_rows = n;
            k.w_every = every;
            k.w_max = o.max_it;
        }
    }
    if (k.whole) {
        KSP_CUDA(cudaGraphLaunch(k.whole, st));
        KSP_CUDA(cudaStreamSynchronize(st));
        ksp_read_host(k, info);
        return OSR_OK;
    }
    solve_prologue<N>(k, p, st);
    KSP_CUDA(cudaGetLastError());
    // the batch graph: every kernel reads its scalars and the solve's status
    // from device memory, so one capture serves every batch of this system
    if (k.batch && (k.g_vals != vals || k.g_x != x || k.g_rows != n || k.g_every != every)) {
        cudaGraphExecDestroy(k.batch);
        k.batch = nullptr;
    }
    if (!k.batch && o.max_it >= every) {
        if (!k.cap) KSP_CUDA(cudaStreamCreateWithFlags(&k.cap, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(k.cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            solve_iterations<N>(k, p, k.cap, every);
            if (cudaStreamEndCapture(k.cap, &graph) == cudaSuccess && graph) {
                if (cudaGraphInstantiate(&k.batch, graph, 0) != cudaSuccess) k.batch = nullptr;
                cudaGraphDestroy(graph);
            }
        }
        cudaGetLastError();   // a failed capture falls back to direct launches
        if (k.batch) {
            k.g_vals = vals;
            k.g_x = x;
            k.g_rows = n;
            k.g_every = every;
        }
    }
    int launched = 0;
    for (;;) {
        if (k.batch && launched + every <= o.max_it) {
            KSP_CUDA(cudaGraphLaunch(k.batch, st));
            launched += every;
        } else {
            const int c = every < o.max_it - launched ? every : o.max_it - launched;
            solve_iterations<N>(k, p, st, c);
            launched += c;
        }
        KSP_CUDA(cudaGetLastError());
        KSP_CUDA(cudaMemcpyAsync(k.host, k.scal, sizeof(osrk::KspScal), cudaMemcpyDeviceToHost, st));
        KSP_CUDA(cudaStreamSynchronize(st));
        if (k.host->reason != osrk::kItersRunning || launched >= o.max_it) break;
    }
    ksp_read_host(k, info);
    return OSR_OK;
}

// The solve with the transposed matrix, J^T x = b (the adjoint system of
// the Newton step): the same left-preconditioned BiCGStab with J^T in the
// products (osr::jacobian_transpose_apply, atomic additions) and the
// transposed inverse blocks as preconditioner; direct launches, the state
// read back every `every` iterations.
template <int N>
static osr_status solve_t_n(osr_grid &g, const double *vals, const double *b, double *x, const osr_ksp_opts &o,
                            osr_ksp_info *info, cudaStream_t st) {
    osr_status rc = ksp_ensure(g);
    if (rc != OSR_OK) return rc;
    osr_ksp_work &k = *g.ksp;
    const SolvePlan<N> p = solve_plan<N>(g, vals, b, x);
    ksp_set_host(k, o);
    const int every = o.check_every > 0 ? o.check_every : 8;
    KSP_CUDA(cudaMemcpyAsync(k.scal, k.host, sizeof(osrk::KspScal), cudaMemcpyHostToDevice, st));
    osrk::bjac_invert_kernel<N><<<p.ib, p.tpb, 0, st>>>(p.v, k.inv, k.scal);
    osrk::bjac_apply_kernel<N, 0, false, true><<<p.ab, p.atb, 0, st>>>(p.v, k.inv, b, k.r, nullptr, k.part, k.scal);
    osrk::bcgs_setup_kernel<<<p.vbk, 256, 0, st>>>(p.n, k.r, k.r0, k.p, k.v, x);
    KSP_CUDA(cudaGetLastError());
    int launched = 0;
    for (;;) {
        const int c = every < o.max_it - launched ? every : o.max_it - launched;
        for (int q = 0; q < c; q++) {
            osrk::bcgs_p_kernel<<<p.vbk, 256, 0, st>>>(p.n, k.r, k.p, k.v, k.scal);
            if ((rc = jacobian_transpose_apply(g, vals, k.p, k.t, st)) != OSR_OK) return rc;
            osrk::bjac_apply_kernel<N, 1, false, true><<<p.ab, p.atb, 0, st>>>(p.v, k.inv, k.t, k.v, k.r0, k.part,
                                                                               k.scal);
            osrk::bcgs_s_kernel<<<p.vbk, 256, 0, st>>>(p.n, k.r, k.v, k.s, k.scal);
            if ((rc = jacobian_transpose_apply(g, vals, k.s, k.w, st)) != OSR_OK) return rc;
            osrk::bjac_apply_kernel<N, 2, false, true><<<p.ab, p.atb, 0, st>>>(p.v, k.inv, k.w, k.t, k.s, k.part,
                                                                               k.scal);
            osrk::bcgs_xr_kernel<<<p.xb, osrk::kRedThreads, 0, st>>>(p.n, x, k.p, k.s, k.t, k.r, k.r0, k.part,
                                                                      k.scal);
        }
        launched += c;
        KSP_CUDA(cudaGetLastError());
        KSP_CUDA(cudaMemcpyAsync(k.host, k.scal, sizeof(osrk::KspScal), cudaMemcpyDeviceToHost, st));
        KSP_CUDA(cudaStreamSynchronize(st));
        if (k.host->reason != osrk::kItersRunning || launched >= o.max_it) break;
    }
    ksp_read_host(k, info);
    return OSR_OK;
}

template <int N>
static osr_status step_graph_n(osr_grid &g, const double *vals, const double *b, double *x, const osr_ksp_opts &o,
                               const std::function<void(cudaStream_t)> &pre,
                               const std::function<void(cudaStream_t)> &post, const GraphExtend *extend,
                               cudaGraphExec_t *out) {
    osr_status rc = ksp_ensure(g);
    if (rc != OSR_OK) return rc;
    const int every = o.check_every > 0 ? o.check_every : 8;
    if (!(o.max_it >= every && o.max_it % every == 0)) return OSR_ERR_UNSUPPORTED;
    const SolvePlan<N> p = solve_plan<N>(g, vals, b, x);
    return build_solve_graph<N>(*g.ksp, p, every, o.max_it, &pre, &post, extend, out) ? OSR_OK : OSR_ERR_CUDA;
}

// The set-up (stage -1) or stage 1..6 of one slab's distributed solve (the
// stage list in ksp_kernels.cuh); stage 0 is the set-up's scalar step.
template <int N>
static osr_status dksp_stage_n(osr_dksp &d, int stage, cudaStream_t st) {
    osr_grid &g = *d.g;
    osr_ksp_work &k = *g.ksp;
    const osrk::KView v = kview(g, d.vals);
    const long n = d.rows, nb = 2 * g.cells;
    const unsigned vbk = vec_blocks(n), ab = red_blocks(nb, osrk::kApplyThreads);
    const unsigned xb = red_blocks(n, 4 * osrk::kRedThreads), atb = osrk::kApplyThreads;
    switch (stage) {
        case -1:
            KSP_CUDA(cudaMemcpyAsync(d.scal, d.host, sizeof(osrk::KspScal), cudaMemcpyHostToDevice, st));
            osrk::bjac_invert_kernel<N><<<inv_blocks(nb), 32 * osrk::kInvWarps, 0, st>>>(v, k.inv, d.scal);
            osrk::bjac_apply_kernel<N, 0, true><<<ab, atb, 0, st>>>(v, k.inv, d.b, k.r, nullptr, k.part, d.scal,
                                                                    d.own, d.dots);
            osrk::bcgs_setup_kernel<<<vbk, 256, 0, st>>>(n, k.r, k.r0, d.p, k.v, d.x);
            break;
        case 0:
            osrk::dksp_scalar_kernel<<<1, 32, 0, st>>>(d.scal, d.dots, 0);
            break;
        case 1:
            osrk::bcgs_p_kernel<<<vbk, 256, 0, st>>>(n, k.r, d.p, k.v, d.scal);
            break;
        case 2:
            spmv_launch<N>(v, d.p, k.t, d.scal, st);
            osrk::bjac_apply_kernel<N, 1, true><<<ab, atb, 0, st>>>(v, k.inv, k.t, k.v, k.r0, k.part, d.scal,
                                                                    d.own, d.dots);
            break;
        case 3:
            osrk::dksp_scalar_kernel<<<1, 32, 0, st>>>(d.scal, d.dots, 3);
            osrk::bcgs_s_kernel<<<vbk, 256, 0, st>>>(n, k.r, k.v, d.s, d.scal);
            break;
        case 4:
            spmv_launch<N>(v, d.s, k.w, d.scal, st);
            osrk::bjac_apply_kernel<N, 2, true><<<ab, atb, 0, st>>>(v, k.inv, k.w, k.t, d.s, k.part, d.scal,
                                                                    d.own, d.dots);
            break;
        case 5:
            osrk::dksp_scalar_kernel<<<1, 32, 0, st>>>(d.scal, d.dots, 5);
            osrk::dbcgs_xr_kernel<<<xb, osrk::kRedThreads, 0, st>>>(n, d.x, d.p, d.s, k.t, k.r, k.r0, g.rowoff,
                                                                    d.own, k.part, d.dots, d.scal);
            break;
        case 6:
            osrk::dksp_scalar_kernel<<<1, 32, 0, st>>>(d.scal, d.dots, 6);
            break;
        default:
            return OSR_ERR_ARG;
    }
    KSP_CUDA(cudaGetLastError());
    return OSR_OK;
}

#define KSP_SWITCH(call)                                                                                  \
    switch (g->nc) {                                                                                      \
        case 1: { constexpr int K = 1; return call; }                                                     \
        case 2: { constexpr int K = 2; return call; }                                                     \
        case 3: { constexpr int K = 3; return call; }                                                     \
        case 4: { constexpr int K = 4; return call; }                                                     \
        case 5: { constexpr int K = 5; return call; }                                                     \
        case 6: { constexpr int K = 6; return call; }                                                     \
        case 7: { constexpr int K = 7; return call; }                                                     \
        case 8: { constexpr int K = 8; return call; }                                                     \
        case 9: { constexpr int K = 9; return call; }                                                     \
        case 10: { constexpr int K = 10; return call; }                                                   \
        case 11: { constexpr int K = 11; return call; }                                                   \
        case 12: { constexpr int K = 12; return call; }                                                   \
        case 13: { constexpr int K = 13; return call; }                                                   \
        case 14: { constexpr int K = 14; return call; }                                                   \
        case 15: { constexpr int K = 15; return call; }                                                   \
        case 16: { constexpr int K = 16; return call; }                                                   \
        default: return OSR_ERR_NC;                                                                       \
    }

osr_status ksp_step_graph(osr_grid &grid, const double *vals, const double *b, double *x, const osr_ksp_opts &o,
                          const std::function<void(cudaStream_t)> &pre, const std::function<void(cudaStream_t)> &post,
                          const GraphExtend *extend, cudaGraphExec_t *out) {
    osr_grid *g = &grid;
    KSP_SWITCH(step_graph_n<K>(grid, vals, b, x, o, pre, post, extend, out))
}

const int *ksp_reason_device(const osr_grid &g) {
    return g.ksp ? (const int *)((const char *)g.ksp->scal + offsetof(osrk::KspScal, reason)) : nullptr;
}

void ksp_step_set_host(osr_grid &g, const osr_ksp_opts &o) {
    if (g.ksp) ksp_set_host(*g.ksp, o);
}

void ksp_step_read_host(const osr_grid &g, osr_ksp_info *info) {
    if (g.ksp) ksp_read_host(*g.ksp, info);
}

}  // namespace osr

extern "C" {

void osr_ksp_default_opts(osr_ksp_opts *o) {
    if (!o) return;
    o->rtol = 1e-18;
    o->atol = 1e-50;
    o->dtol = 1e3;
    o->max_it = 5000;
    o->check_every = 8;
}

osr_status osr_grid_jacobian_apply(osr_grid *g, const double *d_vals, const double *d_x, double *d_y, void *stream) {
    if (!g || !d_vals || !d_x || !d_y || !g->rowoff || g->n_rows <= 0) return OSR_ERR_ARG;
    KSP_SWITCH(osr::spmv_n<K>(*g, d_vals, d_x, d_y, (cudaStream_t)stream))
}

osr_status osr_dksp_create(osr_grid *g, osr_dksp **out) {
    if (!g || !out) return OSR_ERR_ARG;
    osr_status rc = osr::ksp_ensure(*g);
    if (rc != OSR_OK) return rc;
    osr_dksp *d = new osr_dksp();
    d->g = g;
    if (cudaMalloc((void **)&d->scal, sizeof(osrk::KspScal)) != cudaSuccess ||
        cudaMallocHost((void **)&d->host, sizeof(osrk::KspScal)) != cudaSuccess) {
        osr_dksp_destroy(d);
        return OSR_ERR_CUDA;
    }
    *out = d;
    return OSR_OK;
}

void osr_dksp_destroy(osr_dksp *d) {
    if (!d) return;
    if (d->scal) cudaFree(d->scal);
    if (d->host) cudaFreeHost(d->host);
    delete d;
}

osr_status osr_dksp_begin(osr_dksp *d, const double *d_vals, const double *d_b, double *d_x, double *d_p,
                          double *d_s, const long *owned, const osr_ksp_opts *opts, double *d_dots, void *stream) {
    if (!d || !d_vals || !d_b || !d_x || !d_p || !d_s || !owned || !d_dots) return OSR_ERR_ARG;
    osr_grid *g = d->g;
    if (!g->rowoff || g->n_rows <= 0 || !g->ksp) return OSR_ERR_ARG;
    const long nb = 2 * g->cells;
    if (!(0 <= owned[0] && owned[0] <= owned[1] && owned[1] <= g->cells && g->cells <= owned[2] &&
          owned[2] <= owned[3] && owned[3] <= nb))
        return OSR_ERR_ARG;
    osr_ksp_opts o;
    osr_ksp_default_opts(&o);
    if (opts) o = *opts;
    if (o.max_it < 0 || !(o.rtol >= 0) || !(o.atol >= 0)) return OSR_ERR_ARG;
    d->vals = d_vals;
    d->b = d_b;
    d->x = d_x;
    d->p = d_p;
    d->s = d_s;
    d->dots = d_dots;
    d->own.b0 = owned[0];
    d->own.b1 = owned[1];
    d->own.b2 = owned[2];
    d->own.b3 = owned[3];
    d->rows = g->n_rows;
    std::memset(d->host, 0, sizeof(osrk::KspScal));
    d->host->rtol = o.rtol;
    d->host->atol = o.atol;
    d->host->dtol = o.dtol;
    d->host->max_it = o.max_it;
    KSP_SWITCH(osr::dksp_stage_n<K>(*d, -1, (cudaStream_t)stream))
}

osr_status osr_dksp_stage(osr_dksp *d, int stage, void *stream) {
    if (!d || !d->vals || stage < 0 || stage > 6) return OSR_ERR_ARG;
    osr_grid *g = d->g;
    if (g->n_rows != d->rows) return OSR_ERR_ARG;   // the layout changed since osr_dksp_begin
    KSP_SWITCH(osr::dksp_stage_n<K>(*d, stage, (cudaStream_t)stream))
}

osr_status osr_dksp_info(osr_dksp *d, osr_ksp_info *info, void *stream) {
    if (!d || !info) return OSR_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(d->host, d->scal, sizeof(osrk::KspScal), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return OSR_ERR_CUDA;
    info->reason = d->host->reason;
    info->its = d->host->its;
    info->rnorm0 = d->host->rnorm0;
    info->rnorm = d->host->rnorm;
    return OSR_OK;
}

osr_status osr_grid_ksp_solve_transpose(osr_grid *g, const double *d_vals, const double *d_rhs, double *d_sol,
                                        const osr_ksp_opts *opts, osr_ksp_info *info, void *stream) {
    if (!g || !d_vals || !d_rhs || !d_sol || !g->rowoff || g->n_rows <= 0) return OSR_ERR_ARG;
    osr_ksp_opts o;
    osr_ksp_default_opts(&o);
    if (opts) o = *opts;
    if (o.max_it < 0 || !(o.rtol >= 0) || !(o.atol >= 0)) return OSR_ERR_ARG;
    KSP_SWITCH(osr::solve_t_n<K>(*g, d_vals, d_rhs, d_sol, o, info, (cudaStream_t)stream))
}

osr_status osr_grid_ksp_solve(osr_grid *g, const double *d_vals, const double *d_rhs, double *d_sol,
                              const osr_ksp_opts *opts, osr_ksp_info *info, void *stream) {
    if (!g || !d_vals || !d_rhs || !d_sol || !g->rowoff || g->n_rows <= 0) return OSR_ERR_ARG;
    osr_ksp_opts o;
    osr_ksp_default_opts(&o);
    if (opts) o = *opts;
    if (o.max_it < 0 || !(o.rtol >= 0) || !(o.atol >= 0)) return OSR_ERR_ARG;
    KSP_SWITCH(osr::solve_n<K>(*g, d_vals, d_rhs, d_sol, o, info, (cudaStream_t)stream))
}

}  // extern "C"
