// Time stepping on the device: one call of osr_sim_step is one pass of the
// reference's main loop (compsim/PrimeSim.cpp:93-104):
//
//   SolveNonLinear (compsim/PetscAUX.cpp:566-731) with SNESKSPONLY: from the
//   unknowns of the current state (InitGuess2), F(x0) (FormFunction), J(x0)
//   (FormJacobian), one linear solve J dx = F (osr_grid_ksp_solve),
//   x1 = x0 - dx; the step is accepted when the solve converged and
//   |dx|_1 / rows <= TOLMAIN (1e-2) is a number; an accepted step ends with
//   UpdateAll(x1, true) (phase control, PCoeff, PJac, properties) and
//   CreateBackups (compsim/Do_Time_Step.cpp:86-159);
//
//   TimeStepCtrl (compsim/Do_Time_Step.cpp:391-470): after an accepted step
//   the time advances by Dt, Dt grows by 1.03 after every 5 accepted steps
//   (NTIMESTERINC, TIME_STEP_INC), is clamped to [MINDT, DTMAX] and cut to
//   the next time marker (a well's start or end, the total time) when it
//   would pass it or land within 1e-5 s of it; after a rejected step Dt is
//   divided by 1.5 (TIME_STEP_DEC) and the backed-up state (pressures,
//   saturations, phase compositions, labels, well latches) is restored and
//   the row layout rebuilt (RestoreBackups, PJac).  A Dt below MINDT (1e-10 s)
//   ends the run with an error, where the reference terminates.
//
// From the second pass on, the whole pass but TimeStepCtrl runs as one CUDA
// graph: InitGuess2, FormFunction, FormJacobian, the linear solve (its
// iterations a device-side while loop), x1 = x0 - dx and |dx|_1, the
// acceptance test, then a device-side if / else: UpdateAll(x1, true) and
// CreateBackups, or RestoreBackups and PJac.  The kernels read Dt, the time
// and PCoeff from a 3-double device array the graph fills first, so one
// capture serves every pass until the row count changes.  TimeStepCtrl (a
// few host scalars) follows on the host.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "grid_internal.h"
#include "jacobian_kernels.cuh"

namespace {

constexpr double kTolMain = 1e-2;       // TOLMAIN
constexpr double kMinDt = 1e-10;        // MINDT
constexpr double kStepInc = 1.03;       // TIME_STEP_INC
constexpr double kStepDec = 1.5;        // TIME_STEP_DEC
constexpr int kStepsPerInc = 5;         // NTIMESTERINC
constexpr double kMarkerTol = 1e-5;     // TSTEPIF
constexpr int kSumBlocks = 296;

// x <- x - dx and per-CTA partial sums of |dx| (fixed order).
__global__ void __launch_bounds__(256) update_norm1_kernel(long n, double *__restrict__ x,
                                                           const double *__restrict__ dx, double *part) {
    __shared__ double sm[8];
    double a = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double d = dx[i];
        x[i] -= d;
        a += fabs(d);
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sm[w];
        part[blockIdx.x] = t;
    }
}

__global__ void sum_parts_kernel(const double *part, int n, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < n; i++) t += part[i];
        *out = t;
    }
}

// The acceptance test of SolveNonLinear (compsim/PetscAUX.cpp:703): the solve
// converged and |dx|_1 / rows <= TOLMAIN is a number; selects the branch of
// the full step graph (UpdateAll(x, true) + CreateBackups, or RestoreBackups).
__global__ void accept_kernel(cudaGraphConditionalHandle h, const int *reason, const double *sum, double rows,
                              int *flag) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const double vnorm = *sum / rows;
        const bool ok = *reason > 0 && !(vnorm > kTolMain) && vnorm == vnorm;
        *flag = ok ? 1 : 0;
        cudaGraphSetConditional(h, ok ? 1u : 0u);
    }
}

}  // namespace

struct osr_sim {
    osr_grid *g = nullptr;
    double sim_time = 0, dt = 0, max_dt = 0;
    int inc_count = 0, tsm_ctrl = 0;
    std::vector<double> markers;
    long rows_cap = 0;
    double *x = nullptr, *f = nullptr, *dx = nullptr, *vals = nullptr, *part = nullptr;
    double *bP[2] = {nullptr, nullptr}, *bsat[2] = {nullptr, nullptr}, *bx[2] = {nullptr, nullptr},
           *by[2] = {nullptr, nullptr};
    signed char *blab[2] = {nullptr, nullptr};
    std::vector<unsigned char> bcond;
    double *h_sum = nullptr;   // pinned
    // The step graph: InitGuess2, FormFunction, FormJacobian, the whole
    // linear solve and x - dx with |dx|_1, one launch per pass.  Its kernels
    // read the pass's controls [dt, time, PCoeff] from d_ctl, which the graph
    // fills from the pinned h_ctl first; it is captured again when the row
    // layout or the solver options change.
    double *d_ctl = nullptr, *h_ctl = nullptr;
    cudaGraphExec_t graph = nullptr;
    long graph_rows = -1;
    osr_ksp_opts graph_opts{};
    bool use_graph = true, graph_failed = false;
    bool graph_full = false;   // the graph also takes the acceptance and UpdateAll / RestoreBackups
    long graph_launches = 0;
    // what the full graph hands back: PCoeff (bits), row count, acceptance
    struct PassOut {
        unsigned long long pmax;
        long rows;
        int accepted, pad;
    };
    PassOut *h_out = nullptr;   // pinned
    int *d_flag = nullptr;
};

namespace {

#define SIM_CUDA(call)                                     \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return OSR_ERR_CUDA;        \
    } while (0)

void sim_free(osr_sim *s) {
    void *ptrs[] = {s->x, s->f, s->dx, s->vals, s->part, s->bP[0], s->bP[1], s->bsat[0], s->bsat[1],
                    s->bx[0], s->bx[1], s->by[0], s->by[1], s->blab[0], s->blab[1], s->d_ctl, s->d_flag};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (s->h_sum) cudaFreeHost(s->h_sum);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->h_out) cudaFreeHost(s->h_out);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    delete s;
}

bool same_opts(const osr_ksp_opts &a, const osr_ksp_opts &b) {
    return a.rtol == b.rtol && a.atol == b.atol && a.dtol == b.dtol && a.max_it == b.max_it &&
           a.check_every == b.check_every;
}

unsigned norm_blocks(long rows) {
    long nb = (rows + 255) / 256;
    if (nb > kSumBlocks) nb = kSumBlocks;
    if (nb < 1) nb = 1;
    return (unsigned)nb;
}


// CreateBackups / RestoreBackups: the primary state of both continua (device
// copies; capturable).
osr_status copy_state_device(osr_sim &s, bool to_backup, cudaStream_t st) {
    osr_grid &g = *s.g;
    const long n = g.cells, nc = g.nc;
    for (int m = 0; m < 2; m++) {
        const osr::MediumFields &F = g.m[m];
        struct {
            void *live, *bak;
            size_t bytes;
        } items[] = {{F.P, s.bP[m], (size_t)3 * n * 8},
                     {F.sat, s.bsat[m], (size_t)3 * n * 8},
                     {F.x, s.bx[m], (size_t)nc * n * 8},
                     {F.y, s.by[m], (size_t)nc * n * 8},
                     {F.label, s.blab[m], (size_t)n}};
        for (auto &it : items)
            SIM_CUDA(cudaMemcpyAsync(to_backup ? it.bak : it.live, to_backup ? it.live : it.bak, it.bytes,
                                     cudaMemcpyDeviceToDevice, st));
    }
    return OSR_OK;
}

// The well latches of the backup (host side of CreateBackups / RestoreBackups).
osr_status copy_conds(osr_sim &s, bool to_backup) {
    osr_grid &g = *s.g;
    if (to_backup) {
        s.bcond = g.cond_host;
    } else {
        for (int w = 0; w < g.nwells; w++)
            if (g.cond_host[w] != s.bcond[w]) {
                osr_status rc = osr_grid_set_well_condition(&g, w, s.bcond[w]);
                if (rc != OSR_OK) return rc;
            }
    }
    return OSR_OK;
}

osr_status copy_state(osr_sim &s, bool to_backup, cudaStream_t st) {
    osr_status rc = copy_state_device(s, to_backup, st);
    return rc != OSR_OK ? rc : copy_conds(s, to_backup);
}

// Capture the step graph for the current row layout and options.  The
// kernels captured here take the controls from d_ctl (the grid's pointer is
// set for the capture only).  full: the graph also runs the acceptance test
// and, by a device-side if / else, UpdateAll(x, true) + CreateBackups or
// RestoreBackups + PJac, handing PCoeff, the row count and the decision back
// to pinned memory.  False leaves the sim on the shorter graph or on direct
// launches.
bool build_step_graph(osr_sim &s, const osr_ksp_opts &o, bool full) {
    osr_grid *g = s.g;
    const long rows = g->n_rows;
    const unsigned nb = norm_blocks(rows);
    bool fine = true;
    auto pre = [&](cudaStream_t cs) {
        fine = fine && cudaMemcpyAsync(s.d_ctl, s.h_ctl, 3 * sizeof(double), cudaMemcpyHostToDevice, cs) == cudaSuccess;
        fine = fine && osr_grid_init_guess(g, s.x, cs) == OSR_OK;
        fine = fine && osr_grid_form_function(g, s.x, s.f, s.sim_time, cs) == OSR_OK;
        fine = fine && osr_grid_jacobian(g, s.sim_time, s.vals, cs) == OSR_OK;
    };
    auto post = [&](cudaStream_t cs) {
        update_norm1_kernel<<<nb, 256, 0, cs>>>(rows, s.x, s.dx, s.part);
        sum_parts_kernel<<<1, 32, 0, cs>>>(s.part, (int)nb, s.part + kSumBlocks);
        fine = fine && cudaMemcpyAsync(s.h_sum, s.part + kSumBlocks, 8, cudaMemcpyDeviceToHost, cs) == cudaSuccess;
    };
    osr::GraphExtend ext = [&](cudaGraph_t G, cudaStream_t cs, const std::vector<cudaGraphNode_t> &leaves) -> bool {
        const cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, G, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
        if (cudaStreamBeginCaptureToGraph(cs, G, leaves.data(), nullptr, leaves.size(), mode) != cudaSuccess)
            return false;
        accept_kernel<<<1, 32, 0, cs>>>(h, osr::ksp_reason_device(*g), s.part + kSumBlocks, (double)rows, s.d_flag);
        cudaStreamCaptureStatus st2;
        const cudaGraphNode_t *d2 = nullptr;
        size_t n2 = 0;
        bool ok = cudaStreamGetCaptureInfo(cs, &st2, nullptr, nullptr, &d2, &n2) == cudaSuccess &&
                  st2 == cudaStreamCaptureStatusActive;
        std::vector<cudaGraphNode_t> tail(d2, d2 + (ok ? n2 : 0));
        cudaGraph_t tmp = nullptr;
        ok = (cudaStreamEndCapture(cs, &tmp) == cudaSuccess) && ok;
        if (!ok) return false;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 2;   // if: accepted; else: rejected
        cudaGraphNode_t ifnode = nullptr;
        if (cudaGraphAddNode(&ifnode, G, tail.data(), tail.size(), &cp) != cudaSuccess) return false;
        cudaGraph_t acc = cp.conditional.phGraph_out[0], rej = cp.conditional.phGraph_out[1];
        // accepted: UpdateAll(x, true) (unpack, PhaseCtrl, PJac, properties) and CreateBackups
        if (cudaStreamBeginCaptureToGraph(cs, acc, nullptr, nullptr, 0, mode) != cudaSuccess) return false;
        fine = fine && osr::grid_unpack(*g, s.x, cs) == OSR_OK;
        fine = fine && osr_grid_phase_ctrl(g, cs) == OSR_OK;
        fine = fine && osr::relayout_launch(*g, cs) == OSR_OK;
        fine = fine && osr::grid_update(*g, cs) == OSR_OK;
        fine = fine && copy_state_device(s, true, cs) == OSR_OK;
        ok = cudaStreamEndCapture(cs, &tmp) == cudaSuccess;
        // rejected: RestoreBackups and PJac of the restored labels
        if (ok) ok = cudaStreamBeginCaptureToGraph(cs, rej, nullptr, nullptr, 0, mode) == cudaSuccess;
        if (ok) {
            fine = fine && copy_state_device(s, false, cs) == OSR_OK;
            fine = fine && osr::relayout_launch(*g, cs) == OSR_OK;
            ok = cudaStreamEndCapture(cs, &tmp) == cudaSuccess;
        }
        // PCoeff, the row count and the decision back to the host
        if (ok) ok = cudaStreamBeginCaptureToGraph(cs, G, &ifnode, nullptr, 1, mode) == cudaSuccess;
        if (ok) {
            fine = fine && cudaMemcpyAsync(&s.h_out->pmax, g->pmax, 8, cudaMemcpyDeviceToHost, cs) == cudaSuccess;
            fine = fine && cudaMemcpyAsync(&s.h_out->rows, g->rowoff + 2 * g->cells, 8, cudaMemcpyDeviceToHost,
                                           cs) == cudaSuccess;
            fine = fine && cudaMemcpyAsync(&s.h_out->accepted, s.d_flag, 4, cudaMemcpyDeviceToHost, cs) == cudaSuccess;
            ok = cudaStreamEndCapture(cs, &tmp) == cudaSuccess;
        }
        return ok;
    };
    g->d_ctl = s.d_ctl;
    osr_status rc = osr::ksp_step_graph(*g, s.vals, s.f, s.dx, o, pre, post, full ? &ext : nullptr, &s.graph);
    g->d_ctl = nullptr;
    if (rc != OSR_OK || !fine) {
        if (s.graph) cudaGraphExecDestroy(s.graph);
        s.graph = nullptr;
        cudaGetLastError();
        return false;
    }
    s.graph_rows = rows;
    s.graph_opts = o;
    s.graph_full = full;
    return true;
}

}  // namespace

extern "C" {

osr_status osr_sim_create(osr_grid *g, const double *markers, int n_markers, double dt, double max_dt,
                          osr_sim **out) {
    if (!g || !out || !markers || n_markers < 1 || !(dt > 0) || !(max_dt > 0)) return OSR_ERR_ARG;
    *out = nullptr;
    osr_sim *s = new osr_sim();
    s->g = g;
    s->dt = dt;
    s->max_dt = max_dt;
    s->markers.assign(markers, markers + n_markers);
    const long n = g->cells, nc = g->nc;
    s->rows_cap = 2 * n * (2 * nc + 4);
    const long chunks = (2 * n + 31) / 32;
    const size_t vals = (size_t)chunks * osrj::Layout((int)nc).ET * 32;
    cudaError_t e = cudaSuccess;
    auto A = [&](void **p, size_t b) {
        if (e == cudaSuccess) e = cudaMalloc(p, b);
    };
    A((void **)&s->x, s->rows_cap * 8);
    A((void **)&s->f, s->rows_cap * 8);
    A((void **)&s->dx, s->rows_cap * 8);
    A((void **)&s->vals, vals * 8);
    A((void **)&s->part, kSumBlocks * 8 + 8);
    for (int m = 0; m < 2; m++) {
        A((void **)&s->bP[m], 3 * n * 8);
        A((void **)&s->bsat[m], 3 * n * 8);
        A((void **)&s->bx[m], nc * n * 8);
        A((void **)&s->by[m], nc * n * 8);
        A((void **)&s->blab[m], n);
    }
    if (e == cudaSuccess) e = cudaMallocHost((void **)&s->h_sum, 8);
    A((void **)&s->d_ctl, 3 * sizeof(double));
    A((void **)&s->d_flag, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&s->h_ctl, 3 * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&s->h_out, sizeof(osr_sim::PassOut));
    if (e != cudaSuccess) {
        sim_free(s);
        return OSR_ERR_CUDA;
    }
    // the state the caller set is the first backup (UpdateDependencies(true) +
    // CreateBackups before the main loop, compsim/PrimeSim.cpp:85-86)
    osr_status rc = osr_grid_refresh_layout(g, nullptr);
    if (rc == OSR_OK) rc = osr_grid_update_dependencies(g, nullptr);
    if (rc == OSR_OK) rc = copy_state(*s, true, nullptr);
    if (rc == OSR_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) rc = OSR_ERR_CUDA;
    if (rc != OSR_OK) {
        sim_free(s);
        return rc;
    }
    *out = s;
    return OSR_OK;
}

osr_status osr_sim_destroy(osr_sim *s) {
    if (!s) return OSR_ERR_ARG;
    sim_free(s);
    return OSR_OK;
}

osr_status osr_sim_time(osr_sim *s, double *sim_time, double *dt) {
    if (!s) return OSR_ERR_ARG;
    if (sim_time) *sim_time = s->sim_time;
    if (dt) *dt = s->dt;
    return OSR_OK;
}

osr_status osr_sim_marker_index(osr_sim *s, int *tsm_ctrl) {
    if (!s || !tsm_ctrl) return OSR_ERR_ARG;
    *tsm_ctrl = s->tsm_ctrl;
    return OSR_OK;
}

osr_status osr_sim_restart(osr_sim *s, double sim_time, double dt, int tsm_ctrl) {
    if (!s || !(dt > 0) || tsm_ctrl < 0 || tsm_ctrl > (int)s->markers.size()) return OSR_ERR_ARG;
    s->sim_time = sim_time;
    s->dt = dt;
    s->tsm_ctrl = tsm_ctrl;
    s->inc_count = 0;
    // the restored state is the new backup (CreateBackups after ReadRST, compsim/PrimeSim.cpp:84-86)
    osr_status rc = osr_grid_refresh_layout(s->g, nullptr);
    if (rc == OSR_OK) rc = copy_state(*s, true, nullptr);
    if (rc == OSR_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) rc = OSR_ERR_CUDA;
    return rc;
}

osr_status osr_sim_set_graph(osr_sim *s, int on) {
    if (!s) return OSR_ERR_ARG;
    s->use_graph = on != 0;
    s->graph_failed = false;
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    return OSR_OK;
}

osr_status osr_sim_graph_launches(osr_sim *s, long *launches) {
    if (!s || !launches) return OSR_ERR_ARG;
    *launches = s->graph_launches;
    return OSR_OK;
}

osr_status osr_sim_graph_form(osr_sim *s, int *form) {
    if (!s || !form) return OSR_ERR_ARG;
    *form = !s->graph ? 0 : s->graph_full ? 2 : 1;
    return OSR_OK;
}

osr_status osr_sim_step(osr_sim *s, const osr_ksp_opts *opts, osr_step_info *info, void *stream) {
    if (!s) return OSR_ERR_ARG;
    osr_grid *g = s->g;
    cudaStream_t st = (cudaStream_t)stream;
    osr_status rc;
    osr_step_info inf;
    std::memset(&inf, 0, sizeof(inf));
    if (s->tsm_ctrl >= (int)s->markers.size()) {
        inf.finished = 1;
        inf.sim_time = s->sim_time;
        inf.dt = s->dt;
        if (info) *info = inf;
        return OSR_OK;
    }
    // SolveNonLinear
    if ((rc = osr_grid_set_controls(g, s->dt, 0.0)) != OSR_OK) return rc;
    const long rows = g->n_rows;
    inf.rows = rows;
    osr_ksp_opts o;
    osr_ksp_default_opts(&o);
    if (opts) o = *opts;
    osr_ksp_info ki;
    bool graphed = false, full = false;
    if (s->use_graph && !s->graph_failed) {
        if (s->graph && (s->graph_rows != rows || !same_opts(s->graph_opts, o))) {
            cudaGraphExecDestroy(s->graph);
            s->graph = nullptr;
        }
        // the Jacobian's scratch is allocated by its first direct call; the
        // full graph first, the linearisation-and-solve graph if it fails
        if (!s->graph && g->jw_q && !build_step_graph(*s, o, true) && !build_step_graph(*s, o, false))
            s->graph_failed = true;
        if (s->graph) {
            s->h_ctl[0] = s->dt;
            s->h_ctl[1] = s->sim_time;
            s->h_ctl[2] = g->pcoeff;
            osr::ksp_step_set_host(*g, o);
            SIM_CUDA(cudaGraphLaunch(s->graph, st));
            SIM_CUDA(cudaStreamSynchronize(st));
            osr::ksp_step_read_host(*g, &ki);
            s->graph_launches++;
            graphed = true;
            full = s->graph_full;
        }
    }
    if (!graphed) {
        if ((rc = osr_grid_init_guess(g, s->x, stream)) != OSR_OK) return rc;
        if ((rc = osr_grid_form_function(g, s->x, s->f, s->sim_time, stream)) != OSR_OK) return rc;
        if ((rc = osr_grid_jacobian(g, s->sim_time, s->vals, stream)) != OSR_OK) return rc;
        if ((rc = osr_grid_ksp_solve(g, s->vals, s->f, s->dx, &o, &ki, stream)) != OSR_OK) return rc;
        const unsigned nb = norm_blocks(rows);
        update_norm1_kernel<<<nb, 256, 0, st>>>(rows, s->x, s->dx, s->part);
        sum_parts_kernel<<<1, 32, 0, st>>>(s->part, (int)nb, s->part + kSumBlocks);
        SIM_CUDA(cudaGetLastError());
        SIM_CUDA(cudaMemcpyAsync(s->h_sum, s->part + kSumBlocks, 8, cudaMemcpyDeviceToHost, st));
        SIM_CUDA(cudaStreamSynchronize(st));
    }
    inf.ksp_reason = ki.reason;
    inf.ksp_its = ki.its;
    const double vnorm = *s->h_sum / (double)rows;
    inf.vnorm = vnorm;
    const bool accepted = full ? s->h_out->accepted != 0 : (ki.reason > 0 && !(vnorm > kTolMain) && vnorm == vnorm);
    inf.accepted = accepted ? 1 : 0;
    if (full) {
        // the graph ran UpdateAll(x, true) + CreateBackups or RestoreBackups + PJac
        double p;
        std::memcpy(&p, &s->h_out->pmax, 8);
        g->pcoeff = p;
        g->n_rows = s->h_out->rows;
        if ((rc = copy_conds(*s, accepted)) != OSR_OK) return rc;
    } else if (accepted) {
        if ((rc = osr_grid_update_all_full(g, s->x, stream)) != OSR_OK) return rc;
        if ((rc = copy_state(*s, true, st)) != OSR_OK) return rc;
    }
    // TimeStepCtrl
    if (accepted) {
        s->sim_time += s->dt;
        if (++s->inc_count > kStepsPerInc) {
            s->dt *= kStepInc;
            s->inc_count = 0;
        }
        if (s->dt < kMinDt) s->dt = kMinDt;
        if (s->dt > s->max_dt) s->dt = s->max_dt;
        const double mk = s->markers[s->tsm_ctrl];
        if (s->sim_time + s->dt > mk || std::fabs(s->sim_time + s->dt - mk) < kMarkerTol) {
            s->dt = mk - s->sim_time;
            s->tsm_ctrl++;
        }
        if (s->tsm_ctrl == (int)s->markers.size()) inf.finished = 1;
    } else {
        s->inc_count = 0;
        s->dt /= kStepDec;
        if (s->dt < kMinDt) return OSR_ERR_UNSUPPORTED;
        if (!full) {
            if ((rc = copy_state(*s, false, st)) != OSR_OK) return rc;
            if ((rc = osr_grid_refresh_layout(g, stream)) != OSR_OK) return rc;
        }
    }
    SIM_CUDA(cudaStreamSynchronize(st));
    inf.sim_time = s->sim_time;
    inf.dt = s->dt;
    if (info) *info = inf;
    return OSR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// On-disk formats for a C++ host: the restart file (WriteRST / ReadRST,
// compsim/Do_Time_Step.cpp:179-294) and the state listing (PrintAll,
// compsim/ViewAssist.Cpp:39-88).
//
// Restart layout (native little-endian, packed, no header): per continuum
// (matrix, then fracture) the three phase pressures P[Nx+2][Ny+2][Nz+2][3]
// with the one-cell halo (x outermost, the phase innermost; the halo is
// written as zeros -- the reference never writes its edges and corners);
// per continuum, per cell (x outermost, then y, then z) sat[3], then x_i, y_i
// for every component, then the label as one signed byte; then simTime (s),
// Dt (s), TSMCtrl (int32) and SMethQ (double).
// ---------------------------------------------------------------------------
namespace {

struct HostState {
    std::vector<double> P, sat, x, y, z, label;
};

osr_status fetch_state(osr_grid *g, int med, HostState &h) {
    const long n = g->cells;
    const char *m = med ? "f." : "m.";
    h.P.resize(3 * n);
    h.sat.resize(3 * n);
    h.x.resize((size_t)g->nc * n);
    h.y.resize((size_t)g->nc * n);
    h.z.resize((size_t)g->nc * n);
    h.label.resize(n);
    struct {
        const char *k;
        std::vector<double> *v;
    } f[] = {{"P", &h.P}, {"sat", &h.sat}, {"x", &h.x}, {"y", &h.y}, {"z", &h.z}, {"label", &h.label}};
    for (auto &it : f) {
        const std::string name = std::string(m) + it.k;
        osr_status rc = osr_grid_get(g, name.c_str(), it.v->data());
        if (rc != OSR_OK) return rc;
    }
    return OSR_OK;
}

}  // namespace

extern "C" {

osr_status osr_sim_write_restart(osr_sim *s, const char *path, double smethq) {
    if (!s || !path) return OSR_ERR_ARG;
    osr_grid *g = s->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz, nc = g->nc;
    const long n = g->cells;
    HostState st[2];
    for (int m = 0; m < 2; m++) {
        osr_status rc = fetch_state(g, m, st[m]);
        if (rc != OSR_OK) return rc;
    }
    std::vector<unsigned char> buf;
    auto put = [&](const void *p, size_t b) {
        const unsigned char *c = (const unsigned char *)p;
        buf.insert(buf.end(), c, c + b);
    };
    for (int m = 0; m < 2; m++) {
        std::vector<double> halo((size_t)(nx + 2) * (ny + 2) * (nz + 2) * 3, 0.0);
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++)
                for (int iz = 0; iz < nz; iz++) {
                    const long c = ix + (long)nx * (iy + (long)ny * iz);
                    const size_t h = (((size_t)(ix + 1) * (ny + 2) + (iy + 1)) * (nz + 2) + (iz + 1)) * 3;
                    for (int ph = 0; ph < 3; ph++) halo[h + ph] = st[m].P[(size_t)ph * n + c];
                }
        put(halo.data(), halo.size() * 8);
    }
    for (int m = 0; m < 2; m++)
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++)
                for (int iz = 0; iz < nz; iz++) {
                    const long c = ix + (long)nx * (iy + (long)ny * iz);
                    for (int q = 0; q < 3; q++) put(&st[m].sat[(size_t)q * n + c], 8);
                    for (int i = 0; i < nc; i++) {
                        put(&st[m].x[(size_t)i * n + c], 8);
                        put(&st[m].y[(size_t)i * n + c], 8);
                    }
                    const signed char lab = (signed char)st[m].label[c];
                    put(&lab, 1);
                }
    const int tsm = s->tsm_ctrl;
    put(&s->sim_time, 8);
    put(&s->dt, 8);
    put(&tsm, 4);
    put(&smethq, 8);
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return OSR_ERR_ARG;
    const bool ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
    return (std::fclose(fp) == 0 && ok) ? OSR_OK : OSR_ERR_ARG;
}

osr_status osr_sim_read_restart(osr_sim *s, const char *path, double *smethq) {
    if (!s || !path) return OSR_ERR_ARG;
    osr_grid *g = s->g;
    const int nx = g->nx, ny = g->ny, nz = g->nz, nc = g->nc;
    const long n = g->cells;
    const size_t halo = (size_t)(nx + 2) * (ny + 2) * (nz + 2) * 3 * 8, rec = 24 + 16 * (size_t)nc + 1;
    const size_t want = 2 * halo + 2 * rec * (size_t)n + 28;
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return OSR_ERR_ARG;
    std::vector<unsigned char> buf(want + 1);
    const size_t got = std::fread(buf.data(), 1, buf.size(), fp);
    std::fclose(fp);
    if (got != want) return OSR_ERR_ARG;   // not a restart file of this grid and component count
    size_t off = 0;
    auto get = [&](void *p, size_t b) {
        std::memcpy(p, buf.data() + off, b);
        off += b;
    };
    HostState st[2];
    for (int m = 0; m < 2; m++) {
        osr_status rc = fetch_state(g, m, st[m]);   // the overall compositions stay the grid's
        if (rc != OSR_OK) return rc;
    }
    for (int m = 0; m < 2; m++) {
        for (int ix = 0; ix < nx + 2; ix++)
            for (int iy = 0; iy < ny + 2; iy++)
                for (int iz = 0; iz < nz + 2; iz++)
                    for (int ph = 0; ph < 3; ph++) {
                        double v;
                        get(&v, 8);
                        if (ix >= 1 && ix <= nx && iy >= 1 && iy <= ny && iz >= 1 && iz <= nz) {
                            const long c = (ix - 1) + (long)nx * ((iy - 1) + (long)ny * (iz - 1));
                            st[m].P[(size_t)ph * n + c] = v;
                        }
                    }
    }
    std::vector<signed char> labs[2] = {std::vector<signed char>(n), std::vector<signed char>(n)};
    for (int m = 0; m < 2; m++)
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++)
                for (int iz = 0; iz < nz; iz++) {
                    const long c = ix + (long)nx * (iy + (long)ny * iz);
                    for (int q = 0; q < 3; q++) get(&st[m].sat[(size_t)q * n + c], 8);
                    for (int i = 0; i < nc; i++) {
                        get(&st[m].x[(size_t)i * n + c], 8);
                        get(&st[m].y[(size_t)i * n + c], 8);
                    }
                    get(&labs[m][c], 1);
                }
    double t, dt, sm;
    int tsm;
    get(&t, 8);
    get(&dt, 8);
    get(&tsm, 4);
    get(&sm, 8);
    // ReadRST followed by UpdateDependencies(true) (compsim/PrimeSim.cpp:84-85)
    for (int m = 0; m < 2; m++) {
        osr_status rc = osr_grid_set_state(g, m, st[m].P.data() + n, st[m].sat.data(), st[m].x.data(),
                                           st[m].y.data(), st[m].z.data(), labs[m].data(), nullptr);
        if (rc == OSR_OK) rc = osr_grid_set_pressures(g, m, st[m].P.data());
        if (rc != OSR_OK) return rc;
    }
    osr_status rc = osr_grid_phase_ctrl(g, nullptr);
    if (rc == OSR_OK) rc = osr_grid_refresh_layout(g, nullptr);
    if (rc == OSR_OK) rc = osr_grid_update_dependencies(g, nullptr);
    if (rc == OSR_OK) rc = osr_sim_restart(s, t, dt, tsm);
    if (rc == OSR_OK && smethq) *smethq = sm;
    return rc;
}

osr_status osr_grid_write_listing(osr_grid *g, const char *path, double sim_time, int first_call) {
    if (!g || !path) return OSR_ERR_ARG;
    const int nx = g->nx, ny = g->ny, nz = g->nz, nc = g->nc;
    const long n = g->cells;
    HostState st[2];
    for (int m = 0; m < 2; m++) {
        osr_status rc = fetch_state(g, m, st[m]);
        if (rc != OSR_OK) return rc;
    }
    std::string out(80, '-');
    char num[64];
    out += "\n";
    std::snprintf(num, sizeof num, first_call ? "%g" : "%.20g", sim_time / 3600);
    out += num;
    out += "\nX\tY\tZ\tP\t\t\tSw\t\t\tSo\t\t\tSg\t\t\t";
    for (int i = 0; i < nc; i++) out += "Xo[" + std::to_string(i) + "]\t\t\t";
    for (int i = 0; i < nc; i++) out += "Yg[" + std::to_string(i) + "]\t\t\t";
    for (int m = 0; m < 2; m++) {
        out += m ? "\nF\n" : "\nM\n";
        const HostState &h = st[m];
        long c = 0;
        for (int iz = 0; iz < nz; iz++)
            for (int iy = 0; iy < ny; iy++)
                for (int ix = 0; ix < nx; ix++, c++) {
                    char line[256];
                    std::snprintf(line, sizeof line, "\n%d\t%d\t%d\t%.20g\t%.20g\t%.20g\t%.20g", ix, iy, iz, h.P[n + c],
                                  h.sat[c], h.sat[n + c], h.sat[2 * n + c]);
                    out += line;
                    for (int i = 0; i < nc; i++) {
                        std::snprintf(num, sizeof num, "\t%.20g\t", h.x[(size_t)i * n + c]);
                        out += num;
                    }
                    for (int i = 0; i < nc; i++) {
                        std::snprintf(num, sizeof num, "%.20g\t", h.y[(size_t)i * n + c]);
                        out += num;
                    }
                }
    }
    out += "\n\n\n";
    FILE *fp = std::fopen(path, "ab");
    if (!fp) return OSR_ERR_ARG;
    const bool ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
    return (std::fclose(fp) == 0 && ok) ? OSR_OK : OSR_ERR_ARG;
}

}  // extern "C"
