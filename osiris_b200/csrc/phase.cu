// Host side of the phase-appearance step: the saturation pressure of every
// one-phase cell, PhaseCtrl / fPhaseCtrl, and UpdateAll(x, true)
// (compsim/PetscAUX.cpp:176-498 with UpdateDependencies(true), :500-545).
#include <cuda_runtime.h>
#include "grid_internal.h"
#include "phase_kernels.cuh"

namespace osr {

#define PH_CUDA(call)                                  \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return OSR_ERR_CUDA;    \
    } while (0)

template <int N>
static GridArgs<N> phase_args(const osr_grid &g) {
    GridArgs<N> a;
    make_grid_fluid<N>(g, a.g);
    a.s = grid_scalars(g);
    a.geo = GridGeom{g.di, g.dj, g.dk, g.blockH};
    a.m[0] = g.m[0];
    a.m[1] = g.m[1];
    return a;
}

static unsigned phase_blocks(long n) {
    long b = (n + 127) / 128;
    if (b > 148L * 16) b = 148L * 16;
    return (unsigned)(b > 0 ? b : 1);
}

template <int N>
static osr_status sat_pressure_n(osr_grid &g, int med, double *psat, double *xm, cudaStream_t st) {
    sat_pressure_kernel<N><<<phase_blocks(g.cells), 128, 0, st>>>(phase_args<N>(g), med, psat, xm);
    PH_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status phase_ctrl_n(osr_grid &g, cudaStream_t st) {
    phase_ctrl_kernel<N><<<dim3(phase_blocks(g.cells), 2), 128, 0, st>>>(phase_args<N>(g));
    PH_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status sat_pressure_nr_n(osr_grid &g, int med, int kind, double *psat, double *xm, int *status, int *iters,
                                    cudaStream_t st) {
    sat_pressure_nr_kernel<N><<<phase_blocks(g.cells), 128, 0, st>>>(phase_args<N>(g), med, kind, psat, xm, status, iters);
    PH_CUDA(cudaGetLastError());
    return OSR_OK;
}

template <int N>
static osr_status crit_test_n(osr_grid &g, int med, double *lout, int *changed, cudaStream_t st) {
    crit_test_kernel<N><<<phase_blocks(g.cells), 128, 0, st>>>(phase_args<N>(g), med, lout, changed);
    PH_CUDA(cudaGetLastError());
    return OSR_OK;
}

#define PH_SWITCH(call)                                                                                   \
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

osr_status osr_grid_saturation_pressure(osr_grid *g, int medium, double *d_psat, double *d_xm, void *stream) {
    if (!g || !d_psat || (medium != 0 && medium != 1)) return OSR_ERR_ARG;
    PH_SWITCH(sat_pressure_n<K>(*g, medium, d_psat, d_xm, (cudaStream_t)stream))
}

osr_status osr_grid_saturation_pressure_nr(osr_grid *g, int medium, int kind, double *d_psat, double *d_xm,
                                           int *d_status, int *d_iters, void *stream) {
    if (!g || !d_psat || (medium != 0 && medium != 1) || kind < 0 || kind > 2) return OSR_ERR_ARG;
    PH_SWITCH(sat_pressure_nr_n<K>(*g, medium, kind, d_psat, d_xm, d_status, d_iters, (cudaStream_t)stream))
}

osr_status osr_grid_crit_test(osr_grid *g, int medium, double *d_L, int *d_changed, void *stream) {
    if (!g || (medium != 0 && medium != 1)) return OSR_ERR_ARG;
    PH_SWITCH(crit_test_n<K>(*g, medium, d_L, d_changed, (cudaStream_t)stream))
}

osr_status osr_grid_phase_ctrl(osr_grid *g, void *stream) {
    if (!g) return OSR_ERR_ARG;
    PH_SWITCH(phase_ctrl_n<K>(*g, (cudaStream_t)stream))
}

osr_status osr_grid_update_all_full(osr_grid *g, const double *d_x, void *stream) {
    if (!g || !d_x || !(g->pcoeff > 0)) return OSR_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    osr_status s = grid_unpack(*g, d_x, st);
    if (s != OSR_OK) return s;
    if ((s = osr_grid_phase_ctrl(g, stream)) != OSR_OK) return s;
    if ((s = osr_grid_refresh_layout(g, stream)) != OSR_OK) return s;
    return grid_update(*g, st);
}

}  // extern "C"
