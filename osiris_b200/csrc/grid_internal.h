// Internal state of a grid model shared by the grid translation units.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>
#include "osiris_b200.h"
#include "assembly_kernels.cuh"

struct osr_grid {
    int nx, ny, nz, nc, eos;
    long cells;
    double T, wat_ro, wat_mu, refp, cpor, dcpor, lf, re_f, sigma, cdif;
    int const_dif;
    std::vector<double> mw, tc, pc, vc, acf, parachor, zc, kij;
    std::vector<double> swt, sgt;
    std::vector<int> wells_i;
    std::vector<double> wells_f;
    int nwells;
    // device
    char *block = nullptr;
    size_t block_bytes = 0;
    double *di = nullptr, *dj = nullptr, *dk = nullptr, *blockH = nullptr, *d_swt = nullptr, *d_sgt = nullptr;
    double *tor = nullptr;
    osr::MediumFields m[2];
    cudaStream_t stream = nullptr;
    // row layout (PJac) and scaling (CalcPCoeff)
    long *rowoff = nullptr;        // [2 cells + 1]
    long *sizes = nullptr;         // [2 cells]
    unsigned long long *pmax = nullptr;
    long n_rows = 0;
    double pcoeff = 0;
    double dt = 0;
    // per-pass controls [dt, time, PCoeff] in device memory, read by the
    // kernels in place of dt / time / pcoeff when set (osr_sim's step graph)
    const double *d_ctl = nullptr;
    // wells
    int *d_wi = nullptr;
    double *d_wf = nullptr, *d_re = nullptr;
    unsigned char *d_cond = nullptr;
    osr::WellStream *d_ws = nullptr;
    std::vector<double> re_host;
    std::vector<unsigned char> cond_host;
    const double *well_sums_ext = nullptr;   // caller's layer sums of the rate split (osr_grid_set_well_sums)
    // Jacobian scratch: per cell-medium well rates / productivity indices,
    // injection-well index, injected gas compositions, unsupported-cell count
    double *jw_q = nullptr, *jw_pi = nullptr, *j_stream_y = nullptr;
    int *jw_iw = nullptr;
    double *j_dmu = nullptr, *j_dh = nullptr;   // Jacobian derivative tables [2][N+1][2 cells], [2][8+2N][2 cells]
    // linear-solve workspace (ksp.cu), allocated on first use
    struct osr_ksp_work *ksp = nullptr;
};

namespace osr {
GridScalars grid_scalars(const osr_grid &g);
osr_status grid_update(osr_grid &g, cudaStream_t st);
// UpdateAll's unpacking of the unknowns into the state (no property sweeps).
osr_status grid_unpack(osr_grid &g, const double *d_x, cudaStream_t st);
double peaceman_re(const double *di, const double *dj, int nx, int ny, int ix, int iy);
osr_status grid_assembly_init(osr_grid &g, const osr_model *md);
void grid_assembly_free(osr_grid &g);
void ksp_free(osr_grid &g);
// y = J^T x (MatMultTranspose) on the compact Jacobian, y zeroed first.
osr_status jacobian_transpose_apply(const osr_grid &g, const double *vals, const double *x, double *y,
                                    cudaStream_t st);
// PJac / CalcPCoeff launched on `st` without reading the row count and PCoeff
// back (they stay in rowoff[2 cells] and pmax).
osr_status relayout_launch(osr_grid &g, cudaStream_t st);
// The sim's step graph: `pre` (captured ahead), the whole linear solve of
// vals x = b (the reference's KSP options o), the solve's scalars to the
// grid's pinned copy, then `post`, as one instantiated graph.
// `extend` (optional) adds nodes after `post`: it receives the graph, the
// capture stream and the leaf nodes, and returns false on failure.
using GraphExtend = std::function<bool(cudaGraph_t, cudaStream_t, const std::vector<cudaGraphNode_t> &)>;
osr_status ksp_step_graph(osr_grid &g, const double *vals, const double *b, double *x, const osr_ksp_opts &o,
                          const std::function<void(cudaStream_t)> &pre, const std::function<void(cudaStream_t)> &post,
                          const GraphExtend *extend, cudaGraphExec_t *out);
// The scalars the step graph's solve starts from (set before each launch)
// and its outcome (read after the launch has completed).
void ksp_step_set_host(osr_grid &g, const osr_ksp_opts &o);
void ksp_step_read_host(const osr_grid &g, osr_ksp_info *info);
// Device address of the solve's outcome (PETSc KSPConvergedReason; 0 while
// running), valid once the grid's solve workspace exists.
const int *ksp_reason_device(const osr_grid &g);
// Per-component constants at the reservoir temperature, formed with the
// reference's expressions: EOS_Init (compsim/Init_Calcs.cpp:66-97), Tr_Mu
// (:48-64) and the pair factors of CalcDiffusion (compsim/Mass_Tran.cpp:43-46).
template <int N>
inline void make_grid_fluid(const osr_grid &g, GridFluid<N> &G) {
    std::memset(&G, 0, sizeof(G));
    FluidTable<N> &t = G.f;
    t.srk = g.eos == OSR_EOS_SRK;
    double coldia[N], epdia[N];
    for (int i = 0; i < N; i++) {
        double tc = g.tc[i], pc = g.pc[i], w = g.acf[i];
        coldia[i] = 0.1866 * pow(g.vc[i], 1.0 / 3.0) * pow(g.zc[i], -1.2);
        epdia[i] = 65.3 * tc * pow(g.zc[i], 3.6);
        double tr = g.T / tc;
        t.pc[i] = pc;
        t.tc[i] = tc;
        t.wil[i] = 5.37 * (1 + w);
        double ac, m, b;
        if (t.srk) {
            ac = 0.42747 * kR * kR * tc * tc / pc;
            m = 0.48508 + 1.55171 * w - 0.15613 * w * w;
            b = 0.08664 * kR * tc / pc;
        } else {
            ac = 0.457235 * kR * kR * tc * tc / pc;
            m = 0.3796 + 1.485 * w - 0.1644 * w * w + 0.01667 * w * w * w;
            b = 0.077796 * kR * tc / pc;
        }
        t.ac[i] = ac;
        t.m[i] = m;
        t.b[i] = b;
        double a = ac * (1 + m * (1 - sqrt(tr))) * (1 + m * (1 - sqrt(tr)));
        G.sa[i] = sqrt(a);
        for (int j = 0; j < N; j++) t.bic[i * N + j] = 1 - g.kij[i * N + j];
        G.mw[i] = g.mw[i];
        G.smw[i] = sqrt(g.mw[i]);
        double gamma = pow(tc, (1.0 / 6)) / (sqrt(g.mw[i]) * pow((pc / 101325), (2.0 / 3)));
        G.mui[i] = (4.61 * pow(tr, 0.618) - 2.04 * exp(-0.449 * tr) + 1.94 * exp(-4.058 * tr) + 0.1) * 1e-4 / gamma;
        G.vcm[i] = g.vc[i] / 1000000.0;
        G.pcr_atm[i] = pc / 101325;
        G.vc53[i] = pow(G.vcm[i], (5.0 / 3.0));
        G.vc23[i] = pow(G.vcm[i], (2.0 / 3.0));
        G.parachor[i] = g.parachor[i];
    }
    for (int j = 0; j < N; j++) {
        for (int k = 0; k < N; k++) {
            if (j == k) continue;
            double Sij = (coldia[j] + coldia[k]) / 2;
            double Tij = g.T / sqrt(epdia[j] * epdia[k]);
            double Oij = 1.06306 * pow(Tij, -0.1561) + 0.193 * exp(-0.47635 * Tij) + 1.03587 * exp(-1.52996 * Tij) +
                         1.76474 * exp(-3.89411 * Tij);
            G.pD[j * N + k] = 188.2922475 * sqrt(g.T * (1.0 / g.mw[j] + 1.0 / g.mw[k])) / (kR * Oij * Sij * Sij);
            G.pDlast[j] = G.pD[j * N + k];
        }
    }
    G.T = g.T;
}

}  // namespace osr
