// Host side of the Jacobian path: FormJacobian on the device into the
// compact canonical block rows of jacobian_kernels.cuh (values in chunks of
// 32 block rows, [chunk][entry][32]), and the reference (row, column) of
// every value for a COO consumer.
#include <cuda_runtime.h>
#include <cstring>
#include <vector>
#include "grid_internal.h"
#include "jacobian_kernels.cuh"

namespace osr {

static osr_status jfail(cudaError_t) { return OSR_ERR_CUDA; }

#define JAC_CUDA(call)                              \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return jfail(e_);    \
    } while (0)

constexpr int kRowThreads = 128;
// Resident CTAs per SM the row kernels are compiled for (bounds their
// registers): the composition-column kinds (4: 128 registers), the
// pressure-saturation kinds, whose four shared row sums per row and longer
// per-face state spill heavily at 128 registers (3: 168 registers), and the
// fugacity / water / constraint kind, whose per-cell arrays sit in local
// memory anyway and which gains from occupancy (6: 80 registers).  On the
// 128x128x32 PR-8 Jacobian: pressure-saturation kinds at 2 / 3 / 4 CTAs
// 22.9 / 20.8 / 21.9 ms; column kinds at 3 CTAs 22.6 ms; the fugacity kind
// at 3 / 4 / 5 / 6 / 8 CTAs 21.6 / 21.5 / 21.7 / 20.8 / 21.9 ms.
#ifndef OSR_JAC_MIN_BLOCKS
#define OSR_JAC_MIN_BLOCKS 4
#endif
#ifndef OSR_JAC_PS_MIN_BLOCKS
#define OSR_JAC_PS_MIN_BLOCKS 3
#endif
#ifndef OSR_JAC_ROW_MIN_BLOCKS
#define OSR_JAC_ROW_MIN_BLOCKS 6
#endif
constexpr int jac_min_blocks(int kind) {
    return kind == 2 || kind == 3 ? OSR_JAC_PS_MIN_BLOCKS : kind == 4 ? OSR_JAC_ROW_MIN_BLOCKS : OSR_JAC_MIN_BLOCKS;
}

template <int N>
__global__ void __launch_bounds__(kRowThreads) jac_prep_kernel(const __grid_constant__ osrj::JacView v) {
    const long nb = 2 * v.n;
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long)gridDim.x * blockDim.x)
        osrj::prep_cell<N>(v, b);
}

// One warp per (32 consecutive block rows, task) of one kind (see
// jacobian_task_kind): column kinds take tasks k = 0..N-1, the others one
// task.  Each thread's per-row sums: 3N (columns) or 4N (pressure and
// saturations) doubles of dynamic shared memory.
template <int KIND>
__global__ void __launch_bounds__(kRowThreads, jac_min_blocks(KIND)) jacobian_rows_kernel(const __grid_constant__ osrj::JacView v,
                                                                   long chunk0, long chunks) {
    extern __shared__ double s_acc[];
    const int T = KIND <= 1 ? v.nc : 1;
    const int lane = threadIdx.x & 31;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    const long items = chunks * T;
    for (long it = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < items; it += nwarps) {
        const long cq = it / T;
        const int task = (int)(it - cq * T);
        osrj::jacobian_task_kind<KIND>(v, (chunk0 + cq) * 32 + lane, task, s_acc + threadIdx.x, kRowThreads);
    }
}

template <int KIND>
static osr_status launch_rows(const osrj::JacView &v, long chunk0, long chunks, cudaStream_t st) {
    const int tasks = KIND <= 1 ? v.nc : 1;
    const long items = chunks * tasks;
    if (items <= 0) return OSR_OK;
    long rb = (items * 32 + kRowThreads - 1) / kRowThreads;
    if (rb > 148L * 64) rb = 148L * 64;
    const size_t smem = KIND == 4 ? 0 : (size_t)(KIND <= 1 ? 3 : 4) * v.nc * kRowThreads * 8;
    if (smem > 48 * 1024)
        JAC_CUDA(cudaFuncSetAttribute(jacobian_rows_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    jacobian_rows_kernel<KIND><<<(unsigned)rb, kRowThreads, smem, st>>>(v, chunk0, chunks);
    JAC_CUDA(cudaGetLastError());
    return OSR_OK;
}

// Reference (row, column) of every value, in the values' chunked layout.
__global__ void jacobian_pattern_kernel(int N, int nx, int ny, int nz, long n, const long *rowoff,
                                        const signed char *lab_m, const signed char *lab_f, int entries, long *grow,
                                        long *gcol) {
    const long nb = 2 * n, total = (nb + 31) / 32 * 32 * entries;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long chunk = idx / (32L * entries);
        const int e = (int)((idx / 32) % entries);
        const long b = chunk * 32 + (idx & 31);
        long r = -1, c = -1;
        if (b < nb) osrj::entry_position(N, nx, ny, nz, n, rowoff, lab_m, lab_f, b, e, &r, &c);
        grow[idx] = r;
        gcol[idx] = c;
    }
}

template <int N>
static void fill_constants(const osr_grid &g, osrj::JacView &v) {
    GridFluid<N> G;
    make_grid_fluid<N>(g, G);
    for (int i = 0; i < N; i++) {
        v.sa[i] = G.sa[i];
        v.b[i] = G.f.b[i];
        v.mw[i] = G.mw[i];
        v.smw[i] = G.smw[i];
        v.mui[i] = G.mui[i];
        v.vcm[i] = G.vcm[i];
        v.tc[i] = G.f.tc[i];
        v.pc[i] = G.f.pc[i];
        v.pcr_atm[i] = G.pcr_atm[i];
        v.vc53[i] = G.vc53[i];
        v.vc23[i] = G.vc23[i];
        for (int j = 0; j < N; j++) {
            v.bic[i * N + j] = G.f.bic[i * N + j];
            v.pD[i * N + j] = G.pD[i * N + j];
            v.ipD[i * N + j] = 1 / G.pD[i * N + j];
        }
    }
    v.T = G.T;
    v.srk = G.f.srk;
}

static void make_view(const osr_grid &g, osrj::JacView &v) {
    std::memset(&v, 0, sizeof(v));
    v.nx = g.nx;
    v.ny = g.ny;
    v.nz = g.nz;
    v.nc = g.nc;
    v.n = g.cells;
    v.di = g.di;
    v.dj = g.dj;
    v.dk = g.dk;
    v.blockH = g.blockH;
    v.tor = g.tor;
    v.cpor = g.cpor;
    v.dcpor = g.dcpor;
    v.refp = g.refp;
    v.wat_ro = g.wat_ro;
    v.wat_mu = g.wat_mu;
    v.sigma = g.sigma;
    v.lf = g.lf;
    v.pcoeff = g.pcoeff;
    v.dt = g.dt;
    v.ctl = g.d_ctl;
    v.diff_off = (g.const_dif && g.cdif == 0) ? 1 : 0;
    v.const_dif = g.const_dif;
    for (int m = 0; m < 2; m++) {
        const MediumFields &F = g.m[m];
        osrj::JMed &J = v.m[m];
        J.P = F.P;
        J.sat = F.sat;
        J.x = F.x;
        J.y = F.y;
        J.rho = F.rho;
        J.mu = F.mu;
        J.gam = F.gam;
        J.kr = F.kr;
        J.dkr = F.dkr;
        J.pc = F.pc;
        J.dE = F.dE;
        J.diff = F.diff;
        J.trans = F.trans;
        J.wtran = F.wtran;
        J.dwtran = F.dwtran;
        J.por = F.por;
        J.perm = F.perm;
        J.iftran = F.iftran;
        J.label = F.label;
        J.transS = F.transS;
    }
    v.rowoff = g.rowoff;
    v.well_q = g.jw_q;
    v.well_pi = g.jw_pi;
    v.well_comp = g.jw_iw;
    v.stream_y = g.j_stream_y;
    v.dmu = g.j_dmu;
    v.dh = g.j_dh;
}

template <int N>
static osr_status well_pass(osr_grid &g, double sim_time, cudaStream_t st) {
    AsmArgs<N> A;
    A.a.g = GridFluid<N>();
    make_grid_fluid<N>(g, A.a.g);
    A.a.s = grid_scalars(g);
    A.a.geo = GridGeom{g.di, g.dj, g.dk, g.blockH};
    A.a.m[0] = g.m[0];
    A.a.m[1] = g.m[1];
    A.k.dt = g.dt;
    A.k.sim_time = sim_time;
    A.k.pcoeff = g.pcoeff;
    A.k.sigma = g.sigma;
    A.k.lf = g.lf;
    A.k.re_f = g.re_f;
    A.k.diff_off = (g.const_dif && g.cdif == 0) ? 1 : 0;
    A.k.sf1 = A.k.sf3 = 0;
    A.k.ctl = g.d_ctl;
    A.w = WellSet{g.nwells, g.d_wi, g.d_wf, g.d_re, g.d_cond, g.d_ws, g.well_sums_ext};
    A.tor = g.tor;
    A.rowoff = g.rowoff;
    A.f = nullptr;
    A.fscale = nullptr;
    long blocks = (2 * g.cells + 127) / 128;
    if (blocks > 148L * 16) blocks = 148L * 16;
    well_terms_kernel<N><<<(unsigned)blocks, 128, 0, st>>>(A, g.jw_q, g.jw_pi, g.jw_iw);
    JAC_CUDA(cudaGetLastError());
    return OSR_OK;
}

// Well pass, derivative tables, then the row tasks, all on `st`.
template <int N>
static osr_status jacobian_n(osr_grid &g, double sim_time, double *vals, cudaStream_t st) {
    osr_status s = well_pass<N>(g, sim_time, st);
    if (s != OSR_OK) return s;
    osrj::JacView v;
    make_view(g, v);
    fill_constants<N>(g, v);
    v.vals = vals;
    v.entries = osrj::Layout(N).ET;
    const long nb = 2 * g.cells;
    long blocks = (nb + kRowThreads - 1) / kRowThreads;
    if (blocks > 148L * 16) blocks = 148L * 16;
    jac_prep_kernel<N><<<(unsigned)blocks, kRowThreads, 0, st>>>(v);
    JAC_CUDA(cudaGetLastError());
    const long chunks = (nb + 31) / 32, mchunks = (g.cells + 31) / 32, fchunk0 = g.cells / 32;
    if ((s = launch_rows<0>(v, 0, mchunks, st)) != OSR_OK) return s;
    if ((s = launch_rows<1>(v, fchunk0, chunks - fchunk0, st)) != OSR_OK) return s;
    if ((s = launch_rows<2>(v, 0, mchunks, st)) != OSR_OK) return s;
    if ((s = launch_rows<3>(v, fchunk0, chunks - fchunk0, st)) != OSR_OK) return s;
    return launch_rows<4>(v, 0, chunks, st);
}

// y += J^T lambda (MatMultTranspose): every stored value adds value x
// lambda[row] into y[column] of its reference (row, column).  Values that are
// exactly zero are skipped, as a sparse product skips absent entries.  The
// additions into one y entry come from several block rows (atomic adds), so
// the last bits may differ between runs.
__global__ void jacobian_transpose_kernel(int N, int nx, int ny, int nz, long n, const long *rowoff,
                                          const signed char *lab_m, const signed char *lab_f, int entries,
                                          const double *vals, const double *lam, double *y) {
    const long nb = 2 * n, total = (nb + 31) / 32 * 32 * entries;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long chunk = idx / (32L * entries);
        const int e = (int)((idx / 32) % entries);
        const long b = chunk * 32 + (idx & 31);
        if (b >= nb) continue;
        const double v = vals[idx];
        if (v == 0.0) continue;
        long r = -1, c = -1;
        osrj::entry_position(N, nx, ny, nz, n, rowoff, lab_m, lab_f, b, e, &r, &c);
        if (r >= 0 && c >= 0) atomicAdd(y + c, v * lam[r]);
    }
}

// y = J^T x on `st` (y zeroed first).
osr_status jacobian_transpose_apply(const osr_grid &g, const double *vals, const double *x, double *y,
                                    cudaStream_t st) {
    const osrj::Layout L(g.nc);
    JAC_CUDA(cudaMemsetAsync(y, 0, (size_t)g.n_rows * 8, st));
    const long total = (2 * g.cells + 31) / 32 * 32 * L.ET;
    long blocks = (total + 255) / 256;
    if (blocks > 148L * 32) blocks = 148L * 32;
    jacobian_transpose_kernel<<<(unsigned)blocks, 256, 0, st>>>(g.nc, g.nx, g.ny, g.nz, g.cells, g.rowoff,
                                                                g.m[0].label, g.m[1].label, L.ET, vals, x, y);
    JAC_CUDA(cudaGetLastError());
    return OSR_OK;
}

static osr_status ensure_jacobian_scratch(osr_grid &g) {
    if (g.jw_q) return OSR_OK;
    const long nb = 2 * g.cells;
    JAC_CUDA(cudaMalloc((void **)&g.jw_q, nb * 3 * 8));
    JAC_CUDA(cudaMalloc((void **)&g.jw_pi, nb * 3 * 8));
    JAC_CUDA(cudaMalloc((void **)&g.jw_iw, nb * sizeof(int)));
    JAC_CUDA(cudaMalloc((void **)&g.j_dmu, (size_t)nb * 2 * (g.nc + 1) * 8));
    if (!g.const_dif) JAC_CUDA(cudaMalloc((void **)&g.j_dh, (size_t)nb * 2 * (2 * g.nc + 8) * 8));
    const int nw = g.nwells > 0 ? g.nwells : 1;
    JAC_CUDA(cudaMalloc((void **)&g.j_stream_y, (size_t)nw * osrj::kMaxNc * 8));
    JAC_CUDA(cudaMemset(g.j_stream_y, 0, (size_t)nw * osrj::kMaxNc * 8));
    if (g.nwells > 0)
        JAC_CUDA(cudaMemcpy2D(g.j_stream_y, osrj::kMaxNc * 8, (const char *)g.d_ws + offsetof(WellStream, yg),
                              sizeof(WellStream), OSR_MAX_NC * 8, g.nwells, cudaMemcpyDeviceToDevice));
    return OSR_OK;
}

}  // namespace osr

using namespace osr;

extern "C" {

osr_status osr_grid_jacobian_shape(osr_grid *g, int *bs, int *entries, int *overflow) {
    if (!g) return OSR_ERR_ARG;
    const osrj::Layout L(g->nc);
    if (bs) *bs = L.BS;
    if (entries) *entries = L.ET;
    if (overflow) *overflow = osrj::kOverflow;
    return OSR_OK;
}

osr_status osr_grid_block_columns(osr_grid *g, long *out) {
    if (!g || !out) return OSR_ERR_ARG;
    const long n = g->cells;
    for (long b = 0; b < 2 * n; b++) {
        const long med = b >= n, c = med ? b - n : b;
        const int ix = (int)(c % g->nx), iy = (int)((c / g->nx) % g->ny), iz = (int)(c / ((long)g->nx * g->ny));
        long *o = out + 8 * b;
        o[0] = b;
        o[1] = ix > 0 ? b - 1 : -1;
        o[2] = ix < g->nx - 1 ? b + 1 : -1;
        o[3] = iy > 0 ? b - g->nx : -1;
        o[4] = iy < g->ny - 1 ? b + g->nx : -1;
        o[5] = iz > 0 ? b - (long)g->nx * g->ny : -1;
        o[6] = iz < g->nz - 1 ? b + (long)g->nx * g->ny : -1;
        o[7] = med ? c : n + c;
    }
    return OSR_OK;
}

osr_status osr_grid_jacobian_apply_transpose(osr_grid *g, const double *d_vals, const double *d_lambda, double *d_y,
                                            void *stream) {
    if (!g || !d_vals || !d_lambda || !d_y || !g->rowoff || g->n_rows <= 0) return OSR_ERR_ARG;
    return osr::jacobian_transpose_apply(*g, d_vals, d_lambda, d_y, (cudaStream_t)stream);
}

osr_status osr_grid_jacobian_pattern(osr_grid *g, long *d_row, long *d_col, void *stream) {
    if (!g || !d_row || !d_col || !g->rowoff) return OSR_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const osrj::Layout L(g->nc);
    const long total = (2 * g->cells + 31) / 32 * 32 * L.ET;
    long blocks = (total + 255) / 256;
    if (blocks > 148L * 32) blocks = 148L * 32;
    jacobian_pattern_kernel<<<(unsigned)blocks, 256, 0, st>>>(g->nc, g->nx, g->ny, g->nz, g->cells, g->rowoff,
                                                              g->m[0].label, g->m[1].label, L.ET, d_row, d_col);
    JAC_CUDA(cudaGetLastError());
    return OSR_OK;
}

osr_status osr_grid_jacobian(osr_grid *g, double sim_time, double *d_vals, void *stream) {
    if (!g || !d_vals) return OSR_ERR_ARG;
    if (!(g->pcoeff > 0) || !(g->dt > 0)) return OSR_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    osr_status s = ensure_jacobian_scratch(*g);
    if (s != OSR_OK) return s;
    switch (g->nc) {
#define JAC_NC(K) \
    case K: return jacobian_n<K>(*g, sim_time, d_vals, st);
        JAC_NC(1) JAC_NC(2) JAC_NC(3) JAC_NC(4) JAC_NC(5) JAC_NC(6) JAC_NC(7) JAC_NC(8) JAC_NC(9) JAC_NC(10)
        JAC_NC(11) JAC_NC(12) JAC_NC(13) JAC_NC(14) JAC_NC(15) JAC_NC(16)
#undef JAC_NC
        default: return OSR_ERR_NC;
    }
}

osr_status osr_grid_form_jacobian(osr_grid *g, const double *d_x, double sim_time, double *d_vals, void *stream) {
    osr_status s = osr_grid_update_all(g, d_x, stream);
    if (s != OSR_OK) return s;
    return osr_grid_jacobian(g, sim_time, d_vals, stream);
}

}  // extern "C"
