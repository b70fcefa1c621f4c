// Host side of the residual path: row layout, unknown maps, well constants
// and the FormFunction entry points of the C ABI.
#include <cuda_runtime.h>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>
#include "grid_internal.h"

namespace osr {

static osr_status afail(cudaError_t) { return OSR_ERR_CUDA; }

#define ASM_CUDA(call)                              \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return afail(e_);    \
    } while (0)

// Effective radius of a vertical matrix completion from the block's
// neighbour and image-well distances (Calc_Re, compsim/Minor_NR.cpp:2700-3249)
// for a well at the block centre.  Index 1..8 runs over the eight blocks
// around the well block; slots of neighbours outside the reservoir take a
// zero weight, and the image wells mirrored across each reservoir boundary
// enter through their distance ratios.
double peaceman_re(const double *di, const double *dj, int nx, int ny, int ix, int iy) {
    const double dx = di[ix], dy = dj[iy];
    const double xp = 0, yp = 0;   // well position inside the block
    double ri[9], tw[9], rij[5][9], aj[5];
    for (int j = 0; j < 9; j++) {
        ri[j] = 1;
        tw[j] = 0;
        for (int k = 0; k < 5; k++) rij[k][j] = 1;
    }
    for (int k = 0; k < 5; k++) aj[k] = 1;
    auto h = [](double a, double b) { return sqrt(a * a + b * b); };
    ri[1] = h(xp, dy + yp);
    ri[2] = h(dx - xp, yp);
    ri[3] = h(xp, dy - yp);
    ri[4] = h(dx + xp, yp);
    ri[5] = h(dx + xp, dy + yp);
    ri[6] = h(dx - xp, dy + yp);
    ri[7] = h(dx - xp, dy - yp);
    ri[8] = h(dx + xp, dy - yp);
    tw[1] = dx / dy - (tw[5] + tw[6]);
    tw[2] = dy / dx - (tw[6] + tw[7]);
    tw[3] = dx / dy - (tw[7] + tw[8]);
    tw[4] = dy / dx - (tw[5] + tw[8]);
    const double twopi = 2 * 3.1415926535897932384626433;
    double Re = 0;
    auto bsum = [&]() {
        double s = 0;
        for (int j = 1; j < 9; j++) s += tw[j];
        return 1 / s;
    };
    auto drop = [&](std::initializer_list<int> keep, bool images) {
        for (int j = 1; j < 9; j++) {
            bool k = false;
            for (int q : keep) k |= q == j;
            if (!k) {
                tw[j] = 0;
                ri[j] = 1;
                if (images) rij[2][j] = rij[3][j] = rij[4][j] = 1;
            }
        }
    };
    const bool in_x = 0 < ix && ix < nx - 1, in_y = 0 < iy && iy < ny - 1;
    if (in_x && in_y) {  // interior block
        double z = 1;
        for (int j = 1; j < 5; j++) z *= pow(ri[j], tw[j]);
        double b = bsum();
        Re = pow(exp(-twopi * 1) * z, b);
    }
    // a block on one reservoir edge: one image well across that edge
    auto edge = [&](std::initializer_list<int> dropped, double a2) {
        for (int j : dropped) {
            tw[j] = 0;
            ri[j] = 1;
            rij[2][j] = 1;
        }
        aj[2] = a2;
        double b = bsum();
        double z = 1;
        for (int j = 1; j < 5; j++) z *= pow(ri[j], tw[j]) * pow((rij[2][j] / aj[2]), tw[j]);
        Re = pow(exp(-twopi * 1) * z, b);
    };
    if (iy == ny - 1 && ix != 0 && ix != nx - 1) {
        rij[2][2] = h(dx - xp, dy + yp);
        rij[2][7] = h(dx - xp, 2 * dy + yp);
        rij[2][3] = h(xp, 2 * dy + yp);
        rij[2][8] = h(dx + xp, 2 * dy + yp);
        rij[2][4] = h(dx + xp, dy + yp);
        edge({1, 5, 6}, dy + 2 * yp);
    }
    if (iy == 0 && ix != 0 && ix != nx - 1) {
        rij[2][2] = h(dx - xp, dy - yp);
        rij[2][6] = h(dx - xp, 2 * dy - yp);
        rij[2][1] = h(xp, 2 * dy - yp);
        rij[2][5] = h(dx + xp, 2 * dy - yp);
        rij[2][4] = h(dx + xp, dy - yp);
        edge({3, 7, 8}, dy - 2 * yp);
    }
    if (ix == nx - 1 && iy != 0 && iy != ny - 1) {
        rij[2][1] = h(dx - xp, dy + yp);
        rij[2][5] = h(2 * dx - xp, dy + yp);
        rij[2][4] = h(2 * dx - xp, yp);
        rij[2][8] = h(2 * dx - xp, dy - yp);
        rij[2][3] = h(dx - xp, dy - yp);
        edge({2, 7, 6}, dx - 2 * xp);
    }
    if (ix == 0 && iy != 0 && iy != ny - 1) {
        rij[2][1] = h(dx + xp, dy + yp);
        rij[2][7] = h(2 * dx + xp, dy - yp);
        rij[2][2] = h(2 * dx + xp, yp);
        rij[2][6] = h(2 * dx + xp, dy + yp);
        rij[2][3] = h(dx + xp, dy - yp);
        edge({8, 4, 5}, dx + 2 * xp);
    }
    // a corner block: three image wells (across each edge and the corner)
    auto corner = [&](std::initializer_list<int> keep) {
        drop(keep, true);
        double b = bsum();
        double z = 1;
        for (int t = 1; t < 5; t++) {
            double jz = 1;
            for (int j = 2; j < 5; j++) jz *= pow((rij[j][t] / aj[j]), tw[t]);
            z *= pow(ri[t], tw[t]) * jz;
        }
        Re = pow(exp(-twopi * 1) * z, b);
    };
    if (ix == 0 && iy == ny - 1) {
        aj[2] = dy + 2 * yp;
        aj[4] = dx + 2 * xp;
        aj[3] = h(dy + 2 * yp, dx + 2 * xp);
        rij[2][2] = h(dx - xp, dy + yp);
        rij[2][7] = h(dx - xp, 2 * dy + yp);
        rij[2][3] = h(xp, 2 * dy + yp);
        rij[3][2] = h(2 * dx + xp, dy + yp);
        rij[3][3] = h(dx + xp, 2 * dy + yp);
        rij[3][7] = h(2 * dx + xp, 2 * dy + yp);
        rij[4][2] = h(2 * dx + xp, yp);
        rij[4][3] = h(dx + xp, dy - yp);
        rij[4][7] = h(2 * dx + xp, dy - yp);
        corner({2, 3, 7});
    }
    if (ix == 0 && iy == 0) {
        aj[2] = dy - 2 * yp;
        aj[4] = dx + 2 * xp;
        aj[3] = h(dy - 2 * yp, dx + 2 * xp);
        rij[2][2] = h(dx - xp, dy - yp);
        rij[2][6] = h(dx - xp, 2 * dy - yp);
        rij[2][1] = h(xp, 2 * dy - yp);
        rij[3][2] = h(2 * dx + xp, dy - yp);
        rij[3][1] = h(dx + xp, 2 * dy - yp);
        rij[3][6] = h(2 * dx + xp, 2 * dy - yp);
        rij[4][2] = h(2 * dx + xp, yp);
        rij[4][1] = h(dx + xp, dy + yp);
        rij[4][6] = h(2 * dx + xp, dy + yp);
        corner({1, 2, 6});
    }
    if (ix == nx - 1 && iy == ny - 1) {
        aj[2] = dx - 2 * xp;
        aj[4] = dy + 2 * yp;
        aj[3] = h(dx - 2 * xp, dy + 2 * yp);
        rij[2][4] = h(2 * dx - xp, yp);
        rij[2][8] = h(2 * dx - xp, dy - yp);
        rij[2][3] = h(dx - xp, dy - yp);
        rij[3][4] = h(2 * dx - xp, dy + yp);
        rij[3][3] = h(dx - xp, 2 * dy + yp);
        rij[3][8] = h(2 * dx - xp, 2 * dy + yp);
        rij[4][3] = h(2 * dy + yp, xp);
        rij[4][4] = h(dx + xp, dy + yp);
        rij[4][8] = h(dx + xp, 2 * dy + yp);
        corner({3, 4, 8});
    }
    if (ix == nx - 1 && iy == 0) {
        aj[2] = dx - 2 * xp;
        aj[4] = dy - 2 * yp;
        aj[3] = h(dx - 2 * xp, dy - 2 * yp);
        rij[2][1] = h(dx - xp, dy + yp);
        rij[2][5] = h(2 * dx - xp, dy + yp);
        rij[2][4] = h(2 * dx - xp, yp);
        rij[3][4] = h(2 * dx - xp, dy - yp);
        rij[3][1] = h(dx - xp, 2 * dy - yp);
        rij[3][5] = h(2 * dx - xp, 2 * dy - yp);
        rij[4][1] = h(2 * dy - yp, xp);
        rij[4][4] = h(dx + xp, dy - yp);
        rij[4][5] = h(dx + xp, 2 * dy - yp);
        corner({1, 4, 5});
    }
    return Re;
}

template <int N>
static osr_status launch_streams(osr_grid &g) {
    if (g.nwells <= 0) return OSR_OK;
    GridFluid<N> G;
    make_grid_fluid<N>(g, G);
    well_stream_kernel<N><<<(g.nwells + 31) / 32, 32>>>(G, g.nwells, g.d_wi, g.d_wf, g.d_ws);
    ASM_CUDA(cudaGetLastError());
    ASM_CUDA(cudaDeviceSynchronize());
    return OSR_OK;
}

static osr_status dispatch_streams(osr_grid &g) {
    switch (g.nc) {
#define ASM_NC(K) \
    case K: return launch_streams<K>(g);
        ASM_NC(1) ASM_NC(2) ASM_NC(3) ASM_NC(4) ASM_NC(5) ASM_NC(6) ASM_NC(7) ASM_NC(8) ASM_NC(9) ASM_NC(10)
        ASM_NC(11) ASM_NC(12) ASM_NC(13) ASM_NC(14) ASM_NC(15) ASM_NC(16)
#undef ASM_NC
        default: return OSR_ERR_NC;
    }
}

osr_status grid_assembly_init(osr_grid &g, const osr_model *md) {
    const long n = g.cells;
    g.dt = md->dt;
    std::vector<double> tor(n, 1.0);
    if (md->tor) tor.assign(md->tor, md->tor + n);
    ASM_CUDA(cudaMalloc((void **)&g.tor, n * 8));
    ASM_CUDA(cudaMemcpy(g.tor, tor.data(), n * 8, cudaMemcpyHostToDevice));
    ASM_CUDA(cudaMalloc((void **)&g.rowoff, (2 * n + 1) * 8));
    // block sizes, then the scan's chunk sums
    ASM_CUDA(cudaMalloc((void **)&g.sizes, (2 * n + kScanBlocks) * 8));
    ASM_CUDA(cudaMalloc((void **)&g.pmax, 8));
    ASM_CUDA(cudaMemset(g.rowoff, 0, (2 * n + 1) * 8));
    const int nw = g.nwells > 0 ? g.nwells : 0;
    g.re_host.assign(nw, 0.0);
    g.cond_host.assign(nw, 0);
    for (int i = 0; i < nw; i++)
        g.re_host[i] = peaceman_re(md->di, md->dj, g.nx, g.ny, g.wells_i[5 * i + 1], g.wells_i[5 * i + 2]);
    if (nw > 0) {
        ASM_CUDA(cudaMalloc((void **)&g.d_wi, nw * 5 * sizeof(int)));
        ASM_CUDA(cudaMalloc((void **)&g.d_wf, (size_t)nw * (g.nc + 6) * 8));
        ASM_CUDA(cudaMalloc((void **)&g.d_re, nw * 8));
        ASM_CUDA(cudaMalloc((void **)&g.d_cond, nw));
        ASM_CUDA(cudaMalloc((void **)&g.d_ws, nw * sizeof(WellStream)));
        ASM_CUDA(cudaMemcpy(g.d_wi, g.wells_i.data(), nw * 5 * sizeof(int), cudaMemcpyHostToDevice));
        ASM_CUDA(cudaMemcpy(g.d_wf, g.wells_f.data(), (size_t)nw * (g.nc + 6) * 8, cudaMemcpyHostToDevice));
        ASM_CUDA(cudaMemcpy(g.d_re, g.re_host.data(), nw * 8, cudaMemcpyHostToDevice));
        ASM_CUDA(cudaMemcpy(g.d_cond, g.cond_host.data(), nw, cudaMemcpyHostToDevice));
        osr_status st = dispatch_streams(g);
        if (st != OSR_OK) return st;
    }
    return OSR_OK;
}

void grid_assembly_free(osr_grid &g) {
    ksp_free(g);
    void *ptrs[] = {g.tor, g.rowoff, g.sizes, g.pmax, g.d_wi, g.d_wf, g.d_re, g.d_cond, g.d_ws,
                    g.jw_q, g.jw_pi, g.j_stream_y, g.jw_iw, g.j_dmu, g.j_dh};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    g.tor = nullptr;
    g.rowoff = g.sizes = nullptr;
    g.pmax = nullptr;
    g.d_wi = nullptr;
    g.d_wf = g.d_re = nullptr;
    g.d_cond = nullptr;
    g.d_ws = nullptr;
    g.jw_q = g.jw_pi = g.j_stream_y = nullptr;
    g.jw_iw = nullptr;
    g.j_dmu = g.j_dh = nullptr;
}

static long grid_blocks(long work) {
    long b = (work + 127) / 128;
    if (b > 148L * 16) b = 148L * 16;
    if (b < 1) b = 1;
    return b;
}

template <int N>
static GridArgs<N> grid_args(const osr_grid &g) {
    GridArgs<N> a;
    make_grid_fluid<N>(g, a.g);
    a.s = grid_scalars(g);
    a.geo = GridGeom{g.di, g.dj, g.dk, g.blockH};
    a.m[0] = g.m[0];
    a.m[1] = g.m[1];
    return a;
}

template <int N>
static AsmArgs<N> asm_args(const osr_grid &g, double *f, double *fscale, double sim_time) {
    AsmArgs<N> A;
    A.a = grid_args<N>(g);
    A.k.dt = g.dt;
    A.k.sim_time = sim_time;
    A.k.pcoeff = g.pcoeff;
    A.k.sigma = g.sigma;
    A.k.lf = g.lf;
    A.k.re_f = g.re_f;
    A.k.diff_off = (g.const_dif && g.cdif == 0) ? 1 : 0;
    A.k.sf1 = A.k.sf3 = 0;
    A.k.ctl = g.d_ctl;
    A.w = WellSet{g.nwells > 0 ? g.nwells : 0, g.d_wi, g.d_wf, g.d_re, g.d_cond, g.d_ws, g.well_sums_ext};
    A.tor = g.tor;
    A.rowoff = g.rowoff;
    A.f = f;
    A.fscale = fscale;
    return A;
}

template <int N>
static osr_status init_guess_n(osr_grid &g, double *x, cudaStream_t st) {
    GridArgs<N> a = grid_args<N>(g);
    init_guess_kernel<N><<<(unsigned)grid_blocks(2 * g.cells), 128, 0, st>>>(a, g.rowoff, g.pcoeff, g.d_ctl, x);
    ASM_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status update_all_n(osr_grid &g, const double *x, cudaStream_t st) {
    GridArgs<N> a = grid_args<N>(g);
    update_all_kernel<N><<<(unsigned)grid_blocks(2 * g.cells), 128, 0, st>>>(a, g.rowoff, g.pcoeff, g.d_ctl, x);
    ASM_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status residual_n(osr_grid &g, double *f, double *fscale, double t, cudaStream_t st) {
    // the kernel's face tables hold cell indices in 32 bits
    if (2 * g.cells >= (long)INT_MAX) return OSR_ERR_ARG;
    AsmArgs<N> A = asm_args<N>(g, f, fscale, t);
    if (fscale)
        residual_kernel<N, true><<<(unsigned)grid_blocks(2 * g.cells), kResThreads, 0, st>>>(A);
    else
        residual_kernel<N, false><<<(unsigned)grid_blocks(2 * g.cells), kResThreads, 0, st>>>(A);
    ASM_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status logk_vjp_n(osr_grid &g, const double *lam, double *gk, double t, cudaStream_t st) {
    AsmArgs<N> A = asm_args<N>(g, nullptr, nullptr, t);
    residual_logk_vjp_kernel<N><<<(unsigned)grid_blocks(g.cells), 128, 0, st>>>(A, lam, gk);
    ASM_CUDA(cudaGetLastError());
    return OSR_OK;
}

// PJac and CalcPCoeff on the device: block sizes of the current labels, the
// row offsets (multi-CTA scan), the PCoeff maximum into g.pmax.  Row count
// and PCoeff stay on the device (osr_grid_refresh_layout reads them back).
osr_status relayout_launch(osr_grid &g, cudaStream_t st) {
    const long n = g.cells;
    block_size_kernel<<<(unsigned)grid_blocks(2 * n), 128, 0, st>>>(g.m[0].label, g.m[1].label, n, g.nc, g.sizes);
    ASM_CUDA(cudaGetLastError());
    long *part = g.sizes + 2 * n;
    scan_sums_kernel<<<kScanBlocks, kScanThreads, 0, st>>>(g.sizes, 2 * n, part);
    scan_bases_kernel<<<1, 32, 0, st>>>(part, 2 * n, g.rowoff);
    scan_apply_kernel<<<kScanBlocks, kScanThreads, 0, st>>>(g.sizes, 2 * n, part, g.rowoff);
    ASM_CUDA(cudaGetLastError());
    ASM_CUDA(cudaMemsetAsync(g.pmax, 0, 8, st));
    pcoeff_kernel<<<(unsigned)grid_blocks(n), 128, 0, st>>>(g.m[0].P + n, g.m[1].P + n, n, g.pmax);
    ASM_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status well_sums_n(osr_grid &g, int l0, int l1, double *sums, cudaStream_t st) {
    if (g.nwells <= 0) return OSR_OK;
    well_sums_kernel<N><<<(2 * g.nwells + 63) / 64, 64, 0, st>>>(asm_args<N>(g, nullptr, nullptr, 0.0), l0, l1, sums);
    ASM_CUDA(cudaGetLastError());
    return OSR_OK;
}

#define ASM_SWITCH(call)                                                                                  \
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

}  // namespace osr

using namespace osr;

extern "C" {

osr_status osr_grid_refresh_layout(osr_grid *g, void *stream) {
    if (!g) return OSR_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    osr_status rc = osr::relayout_launch(*g, st);
    if (rc != OSR_OK) return rc;
    unsigned long long pm = 0;
    long rows = 0;
    ASM_CUDA(cudaMemcpyAsync(&pm, g->pmax, 8, cudaMemcpyDeviceToHost, st));
    ASM_CUDA(cudaMemcpyAsync(&rows, g->rowoff + 2 * g->cells, 8, cudaMemcpyDeviceToHost, st));
    ASM_CUDA(cudaStreamSynchronize(st));
    double p;
    std::memcpy(&p, &pm, 8);
    g->pcoeff = p;
    g->n_rows = rows;
    return OSR_OK;
}

osr_status osr_grid_layout(osr_grid *g, long *n_rows, double *pcoeff) {
    if (!g) return OSR_ERR_ARG;
    if (n_rows) *n_rows = g->n_rows;
    if (pcoeff) *pcoeff = g->pcoeff;
    return OSR_OK;
}

osr_status osr_grid_row_offsets(osr_grid *g, long *out) {
    if (!g || !out) return OSR_ERR_ARG;
    ASM_CUDA(cudaMemcpy(out, g->rowoff, (2 * g->cells + 1) * 8, cudaMemcpyDeviceToHost));
    return OSR_OK;
}

osr_status osr_grid_set_controls(osr_grid *g, double dt, double pcoeff) {
    if (!g || !(dt > 0)) return OSR_ERR_ARG;
    g->dt = dt;
    if (pcoeff > 0) g->pcoeff = pcoeff;
    return OSR_OK;
}

osr_status osr_grid_set_well_condition(osr_grid *g, int well, int latched) {
    if (!g || well < 0 || well >= g->nwells) return OSR_ERR_ARG;
    g->cond_host[well] = latched ? 1 : 0;
    ASM_CUDA(cudaMemcpy(g->d_cond + well, &g->cond_host[well], 1, cudaMemcpyHostToDevice));
    return OSR_OK;
}

osr_status osr_grid_well_sums(osr_grid *g, int layer0, int layer1, double *d_sums, void *stream) {
    if (!g || !d_sums || layer0 < 0 || layer1 < layer0 || layer1 > g->nz) return OSR_ERR_ARG;
    ASM_SWITCH(well_sums_n<K>(*g, layer0, layer1, d_sums, (cudaStream_t)stream))
}

osr_status osr_grid_set_well_sums(osr_grid *g, const double *d_sums) {
    if (!g) return OSR_ERR_ARG;
    g->well_sums_ext = d_sums;
    return OSR_OK;
}

osr_status osr_grid_well_radius(osr_grid *g, int well, double *re) {
    if (!g || !re || well < 0 || well >= g->nwells) return OSR_ERR_ARG;
    *re = g->re_host[well];
    return OSR_OK;
}

}  // extern "C"

namespace osr {
osr_status grid_unpack(osr_grid &grid, const double *d_x, cudaStream_t st) {
    osr_grid *g = &grid;
    ASM_SWITCH(update_all_n<K>(*g, d_x, st))
}
}  // namespace osr

extern "C" {

osr_status osr_grid_init_guess(osr_grid *g, double *d_x, void *stream) {
    if (!g || !d_x || !(g->pcoeff > 0)) return OSR_ERR_ARG;
    ASM_SWITCH(init_guess_n<K>(*g, d_x, (cudaStream_t)stream))
}

osr_status osr_grid_update_all(osr_grid *g, const double *d_x, void *stream) {
    if (!g || !d_x || !(g->pcoeff > 0)) return OSR_ERR_ARG;
    osr_status s = grid_unpack(*g, d_x, (cudaStream_t)stream);
    if (s != OSR_OK) return s;
    return grid_update(*g, (cudaStream_t)stream);
}

osr_status osr_grid_residual(osr_grid *g, double *d_f, double *d_scale, double sim_time, void *stream) {
    if (!g || !d_f) return OSR_ERR_ARG;
    ASM_SWITCH(residual_n<K>(*g, d_f, d_scale, sim_time, (cudaStream_t)stream))
}

osr_status osr_grid_residual_logk_vjp(osr_grid *g, const double *d_lambda, double *d_gk, double sim_time,
                                      void *stream) {
    if (!g || !d_lambda || !d_gk) return OSR_ERR_ARG;
    ASM_SWITCH(logk_vjp_n<K>(*g, d_lambda, d_gk, sim_time, (cudaStream_t)stream))
}

osr_status osr_grid_form_function(osr_grid *g, const double *d_x, double *d_f, double sim_time, void *stream) {
    osr_status s = osr_grid_update_all(g, d_x, stream);
    if (s != OSR_OK) return s;
    return osr_grid_residual(g, d_f, nullptr, sim_time, stream);
}

}  // extern "C"
