/* osiris_b200: B200-native (sm_100a, FP64 CUDA) per-cell hot path of the
 * Osiris compositional dual-porosity reservoir simulator (khazali/Osiris).
 *
 * C ABI.  Plain pointers and sizes only.  Device pointers are prefixed d_;
 * streams are cudaStream_t passed as void*.  Every entry point returns an
 * osr_status (0 = success) and never exits the process: the reference's fatal
 * paths call TerM() and exit(0) (compsim/Globals.cpp:266-853); here they are
 * status codes.
 *
 * Array layout (structure of arrays, coalesced on the device):
 *   per-cell scalar            [n]
 *   per-component field        [nc][n]        (component-major)
 *   fugacity derivative block  [2][nc][nc][n] (phase, i, k) and [2][nc][n]
 *   phase index 0 = liquid (oil), 1 = vapour (gas).
 * Phase labels follow the reference's phaseStat convention
 * (compsim/Functions.h:327): +1 liquid only, -1 vapour only, 0 two-phase.
 */
#ifndef OSIRIS_B200_H
#define OSIRIS_B200_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OSR_VERSION 1
#define OSR_MAX_NC 16

typedef enum {
    OSR_OK = 0,
    OSR_ERR_ARG = 1,       /* null pointer, n < 0, bad enum */
    OSR_ERR_NC = 2,        /* component count outside 1..OSR_MAX_NC */
    OSR_ERR_CUDA = 3,      /* a CUDA runtime call failed (see osr_last_cuda_error) */
    OSR_ERR_NODEVICE = 4,  /* no sm_100 device is current */
    OSR_ERR_SIZE = 5       /* request larger than the entry point supports */
} osr_status;

typedef enum { OSR_EOS_PR = 0, OSR_EOS_SRK = 1 } osr_eos;

/* Component table (HOST pointers, read during the call only).  Mirrors the
 * reference's fluidProp columns TCRIT, PCRIT, AC and its BIC matrix
 * (compsim/Functions.h:96-111, compsim/Data_Input.cpp:977-990), except that
 * kij is passed directly (the reference stores 1 - kij). */
typedef struct osr_fluid {
    int nc;              /* number of components, 1..OSR_MAX_NC */
    int eos;             /* osr_eos */
    const double *tc;    /* [nc] critical temperature, K */
    const double *pc;    /* [nc] critical pressure, Pa */
    const double *acf;   /* [nc] acentric factor */
    const double *kij;   /* [nc*nc] binary interaction, symmetric, zero diagonal */
} osr_fluid;

/* Outputs of a flash batch (DEVICE pointers).  Required: label, L, x, y, Zl,
 * Zg.  Optional (NULL to skip): iters, rr_iters, dlnphi_dx, dlnphi_dP. */
typedef struct osr_flash_out {
    signed char *label;  /* [n]  +1 / -1 / 0 as phaseStat */
    double *L;           /* [n]  liquid mole fraction after clamping to [0,1] */
    double *x;           /* [nc][n] liquid composition */
    double *y;           /* [nc][n] vapour composition */
    double *Zl, *Zg;     /* [n]  compressibility of each phase (rho = P/(Z R T)) */
    int *iters;          /* [n]  successive-substitution iterations */
    int *rr_iters;       /* [n]  Rachford-Rice Newton iterations, summed */
    double *dlnphi_dx;   /* [2][nc][nc][n] d ln(phi_i)/d w_k, w = x or y */
    double *dlnphi_dP;   /* [2][nc][n]     d ln(phi_i)/d P */
} osr_flash_out;

/* Flash n independent cells at (P, T, z) on the device: the batched,
 * persistent-kernel form.  Replaces the per-cell SuccFalsh/fSuccFalsh calls
 * of AllFlash (compsim/Init_Calcs.cpp:571-738, 740-907, 949-962); the
 * derivative outputs restate the fugacity rows of IteratorJacobian
 * (compsim/Petsc_Functions.cpp:30243-30372).  d_P [n] Pa, d_T [n] K, d_z
 * [nc][n] feed mole fractions.  Asynchronous on `stream` (a cudaStream_t,
 * NULL = legacy default stream).  Takes stream-ordered scratch from a
 * library-private pool per call: work-queue heads and a parked-cell list
 * of (32 + 8 nc) bytes per cell. */
osr_status osr_flash_batch(const osr_fluid *fluid, const double *d_P, const double *d_T, const double *d_z,
                           long n, const osr_flash_out *out, void *stream);

/* Same results as osr_flash_batch, for callers that cannot allocate device
 * memory: a host program embedding the simulator whose device memory is
 * owned by another runtime or allocator (a solver library's pool, a graph
 * being captured by someone else), or that runs under a no-allocation policy
 * in its time-step loop.  The caller passes inputs and outputs as for
 * osr_flash_batch; the work-queue heads and parked-cell lists live in one
 * library-wide static device array of 64 MiB, which every GPU that loads the
 * library holds until the process exits.  No reference counterpart.
 *   - Size limit: n * (48 + 16 * nc) + 4096 bytes must fit in 64 MiB
 *     (about 466,000 cells at nc = 6, 220,000 at nc = 16); larger n returns
 *     OSR_ERR_SIZE before any device work.  Split larger batches.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress, that device current) and caches it; make that
 *     first call before any stream capture.
 *   - Every call shares the array: the call clears its header on `stream`,
 *     and calls that overlap on the GPU (other streams, other threads) race.
 *     Serialise them.
 *   - Calls no cudaMalloc/cudaFree or pool allocation. */
osr_status osr_flash_batch_noalloc(const osr_fluid *fluid, const double *d_P, const double *d_T,
                                   const double *d_z, long n, const osr_flash_out *out, void *stream);

/* Same results, plain form: one thread per cell, no work queue.  Kept as the
 * baseline the batched form is measured against. */
osr_status osr_flash_batch_plain(const osr_fluid *fluid, const double *d_P, const double *d_T,
                                 const double *d_z, long n, const osr_flash_out *out, void *stream);

/* End-to-end form for callers holding HOST arrays (same layouts; out fields
 * are host pointers): copies inputs to the device, runs osr_flash_batch,
 * copies results back, synchronises.  Device buffers come from the
 * stream-ordered pool and are released before return. */
osr_status osr_flash_batch_host(const osr_fluid *fluid, const double *P, const double *T, const double *z,
                                long n, const osr_flash_out *out, void *stream);

/* Launch-shape knobs of the batched flash (the autotuner sets them).
 * The batched form runs two passes of a persistent kernel: the first takes
 * every cell and parks those still running after park_after substitution
 * steps (0 = never park); the second resumes the parked cells, heaviest
 * predicted first.  ss_batch / tail_batch = ready lanes of a warp needed
 * before the substitution step runs in the first / second pass (1..32);
 * ctas_per_sm = persistent CTAs of 128 threads per SM (1..16, capped by
 * occupancy); park_after in 0..500.  Values outside the ranges are
 * rejected.  Process-wide. */
osr_status osr_flash_set_shape(int ss_batch, int tail_batch, int ctas_per_sm, int park_after);
osr_status osr_flash_get_shape(int *ss_batch, int *tail_batch, int *ctas_per_sm, int *park_after);

/* Age limit of the substitution-step batching: a warp runs the step for its
 * ready lanes once they have waited more than max_wait Newton trips, even if
 * fewer than ss_batch/tail_batch lanes are ready (0..1000).  Process-wide. */
osr_status osr_flash_set_max_wait(int max_wait);

/* Measured FP64 FMA-pipe throughput of the current device in TFLOP/s (an FMA
 * counts 2): a dependent-FMA microbenchmark, best of 5 launches.  The
 * denominator of the flash kernel's roofline.  No reference counterpart. */
osr_status osr_probe_fp64_peak(double *tflops, void *stream);

/* Error reporting. */
const char *osr_status_string(osr_status s);
int osr_last_cuda_error(void);
int osr_version(void);

#ifdef __cplusplus
}
#endif
#endif
