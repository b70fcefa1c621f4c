// Host side of the Jacobian path: FormJacobian on the device into a uniform
// block-sparse matrix (block size 2N+4, eight block slots per block row) plus
// a short per-block-row list of entries the reference places outside that
// pattern.
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

__global__ void __launch_bounds__(128) jacobian_kernel(const __grid_constant__ osrj::JacView v, int *unsupported) {
    const long nb = 2 * v.n;
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long)gridDim.x * blockDim.x) {
        if (!osrj::jacobian_block(v, b)) atomicAdd(unsupported, 1);
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
        }
    }
    v.T = G.T;
    v.srk = G.f.srk;
}

static osr_status make_view(const osr_grid &g, osrj::JacView &v) {
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
    switch (g.nc) {
#define JAC_NC(K) \
    case K: fill_constants<K>(g, v); break;
        JAC_NC(1) JAC_NC(2) JAC_NC(3) JAC_NC(4) JAC_NC(5) JAC_NC(6) JAC_NC(7) JAC_NC(8) JAC_NC(9) JAC_NC(10)
        JAC_NC(11) JAC_NC(12) JAC_NC(13) JAC_NC(14) JAC_NC(15) JAC_NC(16)
#undef JAC_NC
        default: return OSR_ERR_NC;
    }
    v.cpor = g.cpor;
    v.dcpor = g.dcpor;
    v.refp = g.refp;
    v.wat_ro = g.wat_ro;
    v.wat_mu = g.wat_mu;
    v.sigma = g.sigma;
    v.lf = g.lf;
    v.pcoeff = g.pcoeff;
    v.dt = g.dt;
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
    v.bs = 2 * g.nc + 4;
    return OSR_OK;
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
    A.w = WellSet{g.nwells, g.d_wi, g.d_wf, g.d_re, g.d_cond, g.d_ws};
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

static osr_status dispatch_well_pass(osr_grid &g, double t, cudaStream_t st) {
    switch (g.nc) {
#define JAC_NC(K) \
    case K: return well_pass<K>(g, t, st);
        JAC_NC(1) JAC_NC(2) JAC_NC(3) JAC_NC(4) JAC_NC(5) JAC_NC(6) JAC_NC(7) JAC_NC(8) JAC_NC(9) JAC_NC(10)
        JAC_NC(11) JAC_NC(12) JAC_NC(13) JAC_NC(14) JAC_NC(15) JAC_NC(16)
#undef JAC_NC
        default: return OSR_ERR_NC;
    }
}

static osr_status ensure_jacobian_scratch(osr_grid &g) {
    if (g.jw_q) return OSR_OK;
    const long nb = 2 * g.cells;
    JAC_CUDA(cudaMalloc((void **)&g.jw_q, nb * 3 * 8));
    JAC_CUDA(cudaMalloc((void **)&g.jw_pi, nb * 3 * 8));
    JAC_CUDA(cudaMalloc((void **)&g.jw_iw, nb * sizeof(int)));
    JAC_CUDA(cudaMalloc((void **)&g.j_unsup, sizeof(int)));
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

osr_status osr_grid_jacobian_shape(osr_grid *g, int *bs, int *slots, int *overflow) {
    if (!g) return OSR_ERR_ARG;
    if (bs) *bs = 2 * g->nc + 4;
    if (slots) *slots = 8;
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

osr_status osr_grid_jacobian(osr_grid *g, double sim_time, const osr_jacobian_out *out, void *stream) {
    if (!g || !out || !out->vals || !out->ovf_row || !out->ovf_col || !out->ovf_val || !out->ovf_n) return OSR_ERR_ARG;
    if (!(g->pcoeff > 0) || !(g->dt > 0)) return OSR_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    osr_status s = ensure_jacobian_scratch(*g);
    if (s != OSR_OK) return s;
    const long nb = 2 * g->cells;
    const int bs = 2 * g->nc + 4;
    JAC_CUDA(cudaMemsetAsync(out->vals, 0, (size_t)nb * 8 * bs * bs * 8, st));
    JAC_CUDA(cudaMemsetAsync(out->ovf_n, 0, (size_t)nb * sizeof(int), st));
    JAC_CUDA(cudaMemsetAsync(g->j_unsup, 0, sizeof(int), st));
    s = dispatch_well_pass(*g, sim_time, st);
    if (s != OSR_OK) return s;
    osrj::JacView v;
    s = make_view(*g, v);
    if (s != OSR_OK) return s;
    v.well_q = g->jw_q;
    v.well_pi = g->jw_pi;
    v.well_comp = g->jw_iw;
    v.stream_y = g->j_stream_y;
    v.vals = out->vals;
    v.ovf_row = out->ovf_row;
    v.ovf_col = out->ovf_col;
    v.ovf_val = out->ovf_val;
    v.ovf_n = out->ovf_n;
    long blocks = (nb + 127) / 128;
    if (blocks > 148L * 16) blocks = 148L * 16;
    jacobian_kernel<<<(unsigned)blocks, 128, 0, st>>>(v, g->j_unsup);
    JAC_CUDA(cudaGetLastError());
    int unsup = 0;
    JAC_CUDA(cudaMemcpyAsync(&unsup, g->j_unsup, sizeof(int), cudaMemcpyDeviceToHost, st));
    JAC_CUDA(cudaStreamSynchronize(st));
    return unsup ? OSR_ERR_UNSUPPORTED : OSR_OK;
}

osr_status osr_grid_form_jacobian(osr_grid *g, const double *d_x, double sim_time, const osr_jacobian_out *out,
                                  void *stream) {
    osr_status s = osr_grid_update_all(g, d_x, stream);
    if (s != OSR_OK) return s;
    return osr_grid_jacobian(g, sim_time, out, stream);
}

}  // extern "C"
