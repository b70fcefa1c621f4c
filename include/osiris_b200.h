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
    OSR_ERR_SIZE = 5,      /* request larger than the entry point supports */
    OSR_ERR_UNSUPPORTED = 6, /* a cell state the entry point does not cover (see its description) */
    OSR_ERR_DECK = 7         /* the deck cannot be read (see osr_deck_error) */
} osr_status;

typedef enum { OSR_EOS_PR = 0, OSR_EOS_SRK = 1 } osr_eos;

/* Per-cell status codes (osr_flash_status, osr_grid_status).  The reference
 * has none: a NaN reaches its acceptance test ((vnorm - vnorm) != 0,
 * compsim/PetscAUX.cpp:703) or its fatal paths (TerM, compsim/Globals.cpp). */
typedef enum {
    OSR_CELL_OK = 0,
    OSR_CELL_MAXIT = 1,   /* the flash's substitution stopped at its 500-step cap */
    OSR_CELL_NAN = 2,     /* a value is not finite */
    OSR_CELL_NOROOT = 3,  /* flash: a present phase's compressibility is not positive */
    OSR_CELL_RANGE = 4    /* grid: oil pressure not positive */
} osr_cell_status;

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
 * library-private pool per call: work-queue heads and two parked-cell lists,
 * 48 + 16 nc bytes per cell in all. */
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
 *     (cudaGetSymbolAddress, that device current) and caches it per CUDA
 *     context; make that first call before any stream capture.  After a
 *     device reset (cudaDeviceReset) or with a new primary context the
 *     next call looks the address up again.
 *   - `stream` must belong to the current device (else OSR_ERR_ARG).
 *   - Every call shares the array: the call clears its header on `stream`,
 *     and calls that overlap on the GPU (other streams, other threads) race.
 *     Serialise them.
 *   - Calls no cudaMalloc/cudaFree or pool allocation. */
osr_status osr_flash_batch_noalloc(const osr_fluid *fluid, const double *d_P, const double *d_T,
                                   const double *d_z, long n, const osr_flash_out *out, void *stream);

/* Many independent instances in one batched call: instance i owns cells
 * [inst_start[i], inst_start[i+1]) of the inputs and outputs and has its own
 * fluid (EOS, criticals, kij); all instances have the same component count.
 * inst_start: HOST [n_inst + 1], inst_start[0] = 0, inst_start[n_inst] = n.
 * Each cell gets exactly the result osr_flash_batch gives it with its own
 * instance's fluid; the work queue spans all instances, so uneven
 * iteration counts across instances are absorbed as within one.  A caller
 * with several component counts makes one call per count. */
osr_status osr_flash_batch_instances(const osr_fluid *fluids, int n_inst, const long *inst_start, const double *d_P,
                                     const double *d_T, const double *d_z, long n, const osr_flash_out *out,
                                     void *stream);

/* A fixed batch of instance groups flashed as one CUDA graph (the batched
 * step of many uneven instances): each group is one osr_flash_batch_instances
 * call's worth (instances of one component count, their cells contiguous).
 * osr_flash_plan_create uploads every group's tables, allocates its scratch
 * and captures all groups' passes and derivative passes, each group on its
 * own branch, into one graph; osr_flash_plan_run is then one graph launch
 * that gives every cell exactly osr_flash_batch_instances's result (the same
 * kernels and launch shapes).  The groups' device pointers (inputs, outputs)
 * are kept by the plan: refill the inputs in place between runs.  Host
 * arrays are read during create only. */
typedef struct {
    const osr_fluid *fluids;    /* HOST [n_inst], one component count */
    int n_inst;
    const long *inst_start;     /* HOST [n_inst + 1], cells of each instance */
    const double *d_P, *d_T, *d_z;
    long n;                     /* cells of the group */
    const osr_flash_out *out;   /* HOST struct of DEVICE outputs */
} osr_flash_group;
typedef struct osr_flash_plan osr_flash_plan;
osr_status osr_flash_plan_create(const osr_flash_group *groups, int n_groups, osr_flash_plan **out);
osr_status osr_flash_plan_run(osr_flash_plan *plan, void *stream);
/* The same step as ONE persistent cooperative kernel launch: every group's
 * passes and derivative pass are work items of a device-side work table
 * (pass p + 1 of a group opens when pass p has no cell left and no CTA in
 * it), taken by whichever CTA is free; each item runs the same pass body as
 * the separate launches, so the results equal osr_flash_plan_run's bit for
 * bit.  Waits for an item are bounded: past the bound the launch records
 * an error (osr_flash_plan_persistent_error) and ends.  OSR_ERR_UNSUPPORTED
 * when the plan has more than 16 groups or the group form is enabled
 * (osr_flash_set_group_from) for a pass the plan runs. */
osr_status osr_flash_plan_run_persistent(osr_flash_plan *plan, void *stream);
/* 1 when a persistent run's wait for a work item ran past its bound
 * (synchronises `stream`). */
osr_status osr_flash_plan_persistent_error(osr_flash_plan *plan, int *error, void *stream);
void osr_flash_plan_destroy(osr_flash_plan *plan);

/* Same results, plain form: one thread per cell, no work queue.  Kept as the
 * baseline the batched form is measured against. */
osr_status osr_flash_batch_plain(const osr_fluid *fluid, const double *d_P, const double *d_T,
                                 const double *d_z, long n, const osr_flash_out *out, void *stream);

/* Fugacity-coefficient derivatives of both phases at given states (DEVICE
 * pointers): d ln(phi_i)/d w_k into d_dlnphi_dx [2][nc][nc][n] and
 * d ln(phi_i)/d P into d_dlnphi_dP [2][nc][n], phase 0 at (d_P, d_T, d_x
 * [nc][n], d_Zl), phase 1 at (d_P, d_T, d_y [nc][n], d_Zg).  The pass the
 * flash runs on its own outputs, for a caller whose compositions come from
 * elsewhere (the reference renormalises them when it unpacks the unknowns,
 * compsim/PetscAUX.cpp:176-498).  Replaces the mixing-rule and implicit-dZ
 * part of the fugacity rows of IteratorJacobian
 * (compsim/Petsc_Functions.cpp:30243-30372).  Asynchronous on `stream`. */
osr_status osr_fugacity_derivs(const osr_fluid *fluid, const double *d_P, const double *d_T, const double *d_x,
                               const double *d_y, const double *d_Zl, const double *d_Zg, long n, double *d_dlnphi_dx,
                               double *d_dlnphi_dP, void *stream);

/* Adjoint of the flash (DEVICE pointers): sensitivities of a flash result
 * to the binary-interaction coefficients, the feed and the pressure.  The
 * reference has no adjoint; this differentiates the equilibrium its
 * SuccFalsh converges to (compsim/Init_Calcs.cpp:571-738) by the implicit
 * function theorem: for a two-phase cell the equal-fugacity, material-
 * balance and Rachford-Rice equations in (x, y, L), an (nc+1) x (nc+1)
 * solve per cell.  `state` holds the flash's outputs for these inputs
 * (label, L, x, y, Zl, Zg; other fields unused); d_xbar, d_ybar [nc][n] and
 * d_Lbar [n] are cotangents on x, y, L.  Outputs: d_kij_bar [nc*nc] =
 * d(sum of cotangent . result)/d k_ij summed over the cells (overwritten;
 * the sum is deterministic), optional d_z_bar [nc][n] and d_P_bar [n].
 * One-phase cells: the present phase equals the feed, so its cotangent goes
 * to z_bar and nothing else; the incipient phase's composition (the
 * reference's unconverged two-step estimate) carries no sensitivity.  Cells
 * whose system is singular (a critical point) contribute nothing and are
 * counted in *singular (may be NULL; when given the call synchronises
 * `stream`).  Two-phase cells that stopped at the 500-step cap are not at
 * the equilibrium and get its sensitivity.  Scratch: blocks x nc^2 doubles
 * from the library pool. */
osr_status osr_flash_adjoint(const osr_fluid *fluid, const double *d_P, const double *d_T, const double *d_z, long n,
                             const osr_flash_out *state, const double *d_xbar, const double *d_ybar,
                             const double *d_Lbar, double *d_kij_bar, double *d_z_bar, double *d_P_bar,
                             long *singular, void *stream);

/* Per-cell status of a flash result (DEVICE `out` of osr_flash_batch for n
 * cells of nc components; iters optional -- without it MAXIT is not
 * detected): d_status [n] (optional) receives an osr_cell_status per cell,
 * counts [4] (HOST) the number of cells per code OK/MAXIT/NAN/NOROOT, and
 * *first_bad (HOST) the lowest cell index whose code is not OK, or -1.
 * Synchronises `stream`. */
osr_status osr_flash_status(const osr_flash_out *out, int nc, long n, signed char *d_status, long *counts,
                            long *first_bad, void *stream);

/* End-to-end form for callers holding HOST arrays (same layouts; out fields
 * are host pointers): the cells go through in chunks of about 131,072
 * (at most 16 chunks) pipelined over three internal streams -- inputs in,
 * osr_flash_batch, results out -- so transfers overlap the flash (pinned
 * host memory gives the overlap; pageable memory works, without it).
 * Results are those of osr_flash_batch.  Waits for the caller's earlier
 * work on `stream` and synchronises before return.  Device buffers come
 * from the stream-ordered pool and are released before return. */
osr_status osr_flash_batch_host(const osr_fluid *fluid, const double *P, const double *T, const double *z,
                                long n, const osr_flash_out *out, void *stream);

/* The host pipeline of osr_flash_batch_host: batches are cut into chunks of
 * about chunk_cells cells (at most 64 chunks), each copied in, flashed and
 * copied out on one of `streams` streams (1..8) in turn, so copies of one
 * chunk overlap the flash of others.  Defaults: 4 streams, 131,072 cells
 * (the best of a sweep of 2-8 streams and 32k-256k cells on the 1M-cell
 * SRK-6 batch with derivatives: 21.1 ms against 23.7 ms for 3 streams). */
osr_status osr_flash_set_host_pipeline(int streams, long chunk_cells);
osr_status osr_flash_get_host_pipeline(int *streams, long *chunk_cells);

/* Launch-shape knobs of the batched flash (the autotuner sets them).
 * The batched form runs a sequence of passes of a persistent kernel: the
 * first takes every cell and parks those still running after park_after
 * substitution steps (0 = never park, one pass); each later pass resumes the
 * parked cells with a doubled limit, up to the reference's 500 steps.
 * ss_batch / tail_batch = ready lanes of a warp needed before the
 * substitution step runs in the first / later passes (1..32);
 * ctas_per_sm = persistent CTAs of 128 threads per SM (1..16, capped by
 * occupancy); park_after in 0..500.  Values outside the ranges are
 * rejected.  Process-wide. */
osr_status osr_flash_set_shape(int ss_batch, int tail_batch, int ctas_per_sm, int park_after);

/* First pass (0-based) of the batched flash that runs in pair form: two
 * lanes per cell, one per phase, for the few long-running cells of the late
 * passes (each substitution step's latency halves).  Default 6 (cells past
 * 64 steps); 12 or more = never.  Process-wide; the results agree to
 * rounding either way. */
osr_status osr_flash_set_pair_from(int pass);
int osr_flash_get_pair_from(void);

/* First pass in group form: one lane per component (2, 4, 8 or 16 lanes per
 * cell), for the last passes, whose few thousand cells run hundreds of
 * steps each with most of the GPU idle.  Takes precedence over the pair
 * form from that pass on.  12 or more = never.  Process-wide. */
osr_status osr_flash_set_group_from(int pass);
int osr_flash_get_group_from(void);
osr_status osr_flash_get_shape(int *ss_batch, int *tail_batch, int *ctas_per_sm, int *park_after);

/* The project's autotuner of the batched flash's launch shape.  Runs every
 * candidate (substitution-step batch 24/28 ready lanes, park after 1/2/3
 * steps, pair form from pass 4/5/6/never, 2/3 CTAs per SM: 48 shapes) on the
 * caller's batch (DEVICE inputs and outputs as osr_flash_batch; the outputs
 * are written), timed with CUDA events on `stream`; keeps the fastest for the
 * batch's (component count, floor(log2 n)) bucket and makes it the current
 * knobs.  No reference counterpart. */
typedef struct osr_flash_tuning {
    int ss_batch, tail_batch, ctas_per_sm, park_after, pair_from;
    float ms;          /* the winner's time per call */
    int candidates;    /* shapes timed */
} osr_flash_tuning;
osr_status osr_flash_autotune(const osr_fluid *fluid, const double *d_P, const double *d_T, const double *d_z,
                              long n, const osr_flash_out *out, void *stream, osr_flash_tuning *best);
/* Use the tuned shape of a call's (component count, size bucket) when one is
 * known (1), or the process-wide knobs always (0, the default). */
osr_status osr_flash_use_tuned(int on);
/* Persist / restore the tuned shapes (a text file, one line per bucket). */
osr_status osr_flash_tuning_save(const char *path);
osr_status osr_flash_tuning_load(const char *path);

/* Age limit of the substitution-step batching: a warp runs the step for its
 * ready lanes once they have waited more than max_wait Newton trips, even if
 * fewer than ss_batch/tail_batch lanes are ready (0..1000).  Process-wide. */
osr_status osr_flash_set_max_wait(int max_wait);

/* ---------------------------------------------------------------------------
 * Grid path: a dual-porosity (matrix + fracture) model on the device.
 * ------------------------------------------------------------------------- */

/* The content of a Data_Input deck (compsim/Data_Input.cpp:13-1349), HOST
 * pointers read during osr_grid_create only.  Cell index c = i + nx*(j +
 * ny*k); per-direction fields are [3][cells] (x, y, z). */
typedef struct osr_model {
    int nx, ny, nz;       /* GRID */
    int nc;               /* NC (pure + pseudo components) */
    int eos;              /* MODEL: osr_eos */
    double restemp;       /* RESTEMP in K (deck value + 273.15) */
    double wat_ro, wat_mu;   /* WATERPROPS */
    double refp, cpor, dcpor;   /* REFP, CPOR, DCPOR */
    double lf, re_f, sigma;     /* Lf, Re_f, SIGMA (1 when absent) */
    int has_cdif;         /* CDIF keyword present */
    double cdif;          /* its value */
    const double *di, *dj, *dk;   /* [nx], [ny], [nz] block sizes, m */
    const double *por, *fpor;     /* [cells] matrix / fracture porosity */
    const double *perm, *fperm;   /* [3][cells] permeability, mD */
    const double *mw, *tc, *pc, *vc, *acf, *parachor, *zc;  /* [nc]; vc in cm3/mol as in the deck */
    const double *kij;            /* [nc*nc] BIC values as listed in the deck (the reference stores 1 - kij) */
    int nswt, nsgt;
    const double *swt, *sgt;      /* [n][4]: S, kr, kro, Pc (SWT: water, SGT: gas) */
    int nwells;
    const int *wells_i;           /* [nwells][5] type, i, j, k0, k1 (0-based, as the reference stores them) */
    const double *wells_f;        /* [nwells][nc+6] the well's values (times in s) */
    const double *tor;            /* [cells] TOR tortuosity, NULL = 1 */
    double dt;                    /* time-step length in s (DT x 3600) */
} osr_model;

typedef struct osr_grid osr_grid;

/* ---------------------------------------------------------------------------
 * Decks: the reference's Data_Input keyword format read in C++
 * (compsim/Data_Input.cpp:13-1349, compsim/MIfstream.cpp:8-47): GRID NC
 * RESTEMP WATERPROPS DI DJ DK TOR POR CDIF SIGMA DTMAX FPOR Lf Re_f PERMI/J/K
 * FPERMI/J/K REFP CPOR DCPOR MODEL SG TB MW AC PCRIT TCRIT VCRIT ZCRIT
 * COMPNAME (the reference's component library) BIC SWT SGT INITCOND 0/1/3
 * with IPRESS FIPRESS IWS FIWS IGC FIGC, WELLS, DT, TOTALT; CON/VAR/IVAR/KVAR
 * arrays and k*v repeat groups.  Host memory only; no device work. */
typedef struct osr_deck osr_deck;

/* Parse a deck file.  OSR_ERR_DECK with the reason in osr_deck_error() when
 * a required keyword is missing or malformed (the reference stops with TerM
 * there, compsim/Data_Input.cpp). */
osr_status osr_deck_open(const char *path, osr_deck **out);
const char *osr_deck_error(void);
/* The parsed values as an osr_model (pointers into the deck, valid until
 * osr_deck_close), ready for osr_grid_create. */
osr_status osr_deck_model(const osr_deck *deck, osr_model *out);
/* The INITCOND state of one medium (0 matrix, 1 fracture): oil pressure
 * [cells], water saturation [cells], feed composition [nc][cells]. */
osr_status osr_deck_initial_state(const osr_deck *deck, int medium, const double **p0, const double **sw0,
                                  const double **z0);
/* DT and TOTALT in s, DTMAX, the INITCOND mode (any may be null). */
osr_status osr_deck_times(const osr_deck *deck, double *dt, double *total_time, double *dtmax, int *initcond);
osr_status osr_deck_close(osr_deck *deck);

/* Open a deck and form the reference's start-up state on the current device
 * (compsim/PrimeSim.cpp:68-85): the INITCOND pressures, water saturations
 * and feed compositions, a flash of every cell-medium (AllFlash,
 * compsim/Init_Calcs.cpp:949-962), then UpdateDependencies(true) (phase
 * control, PCoeff, the row layout, the property sweeps;
 * compsim/PetscAUX.cpp:500-545).  The grid is then ready for
 * osr_grid_form_function / osr_grid_form_jacobian (FormFunction /
 * FormJacobian) and osr_sim_create.  Synchronises `stream` before return;
 * release with osr_grid_destroy. */
osr_status osr_create(const char *deck_path, void *stream, osr_grid **out);

/* Upload a model; geometric transmissibilities (IFK_Calc,
 * compsim/Init_Calcs.cpp:21-46) and block heights are formed here. */
osr_status osr_grid_create(const osr_model *model, osr_grid **out);
osr_status osr_grid_destroy(osr_grid *grid);
osr_status osr_grid_dims(osr_grid *grid, int *dims /* [4]: nx, ny, nz, nc */);

/* Set the state of one medium (0 = matrix, 1 = fracture) from HOST arrays:
 * oil pressure [cells], saturations [3][cells] (water, oil, gas), liquid,
 * vapour and feed compositions [nc][cells], phase labels [cells], and
 * optionally the densities of the previous property update [2][cells]
 * (the interfacial tension is formed from them, as the reference does). */
osr_status osr_grid_set_state(osr_grid *grid, int medium, const double *P_oil, const double *sat, const double *x,
                              const double *y, const double *z, const signed char *label, const double *rho);

/* All three phase pressures of one continuum, HOST [3][cells] (water, oil,
 * gas): what the reference's ReadRST restores (compsim/Do_Time_Step.cpp:
 * 236-260); PhaseCtrl reads the gas pressure before the next update. */
osr_status osr_grid_set_pressures(osr_grid *grid, int medium, const double *P);

/* The property sweeps of UpdateDependencies (compsim/PetscAUX.cpp:530-548)
 * for both media: IFT, relative permeability and capillary pressure, phase
 * pressures, densities with d rho/dx and d rho/dP, LBC viscosities,
 * accumulation at the linearisation point, diffusion coefficients, phase
 * gravity, and the upstream-weighted face transmissibilities. */
osr_status osr_grid_update_dependencies(osr_grid *grid, void *stream);

/* Copy a device field to HOST memory as doubles: "m.<name>" (matrix) or
 * "f.<name>" (fracture), names P sat x y z label rho pc mu gam kr dkr dE pre
 * diff ift trans transS wtran dwtran por perm iftran, laid out [planes][cells].
 * osr_grid_field_size returns planes*cells (or -1 for an unknown name). */
long osr_grid_field_size(osr_grid *grid, const char *field);
osr_status osr_grid_get(osr_grid *grid, const char *field, double *out);

/* State check: *code = OSR_CELL_NAN when any pressure, saturation or phase
 * composition of either continuum is not finite, else OSR_CELL_RANGE when an
 * oil pressure is not positive, else OSR_CELL_OK; *first_bad_block = the
 * lowest such block (matrix blocks 0..cells-1, then fracture), or -1.  Where
 * the reference would run on into its acceptance test or TerM(), a caller
 * can stop first.  Synchronous. */
osr_status osr_grid_status(osr_grid *grid, int *code, long *first_bad_block);

/* ---------------------------------------------------------------------------
 * Residual path: the PETSc FormFunction callback on the device.
 *
 * Row layout (PJac, compsim/Init_Calcs.cpp:1013-1116): blocks of all matrix
 * cells in cell order, then all fracture cells.  A two-phase cell owns 2N+4
 * rows and unknowns [x (N) | y (N), P/PCoeff, Sw, So, Sg]; a one-phase cell N+3
 * [w (N), P/PCoeff, Sw, S of its phase].  Residual rows of a two-phase cell:
 * N fugacity equalities, N-1 component balances, total hydrocarbon, water,
 * sum x - 1, sum y - 1, sum S - 1; of a one-phase cell: N-1 component
 * balances, total, water, sum w - 1, sum S - 1.
 * ------------------------------------------------------------------------- */

/* Row offsets of the current phase labels and the pressure scale PCoeff
 * (the FullTimeStep part of UpdateDependencies: CalcPCoeff and PJac,
 * compsim/PetscAUX.cpp:502-507).  Synchronises `stream`. */
osr_status osr_grid_refresh_layout(osr_grid *grid, void *stream);
osr_status osr_grid_layout(osr_grid *grid, long *n_rows, double *pcoeff);
osr_status osr_grid_row_offsets(osr_grid *grid, long *out /* HOST [2 cells + 1] */);

/* Time-step length (the reference's Dt, seconds) and, when pcoeff > 0, an
 * explicit pressure scale. */
osr_status osr_grid_set_controls(osr_grid *grid, double dt, double pcoeff);

/* The WellCondition latch of a rate-controlled well (switches it to its
 * bottom-hole-pressure limit; compsim/Do_Cycle.cpp:1745). */
osr_status osr_grid_set_well_condition(osr_grid *grid, int well, int latched);

/* Effective radius of the well's matrix completions (Calc_Re,
 * compsim/Minor_NR.cpp:2700-3249), formed once per well at create. */
osr_status osr_grid_well_radius(osr_grid *grid, int well, double *re);

/* Sums over a well's completed layers, both continua, that split the rate of
 * a rate-controlled well (or a latched one) over its completions inside the
 * well regions of IteratorFunction (compsim/Petsc_Functions.cpp:164-702,
 * 3505-4044), taken over this grid's layers [layer0, layer1) at the current
 * state: d_sums DEVICE [nwells][2 completion continua][5].  A z-slab run
 * takes them over each rank's owned layers, adds them over the ranks and
 * hands the totals to osr_grid_set_well_sums, so that a well crossing slabs
 * sees the same sums as on one grid.  Asynchronous. */
osr_status osr_grid_well_sums(osr_grid *grid, int layer0, int layer1, double *d_sums, void *stream);

/* Residual and Jacobian take the wells' layer sums from d_sums (DEVICE, the
 * layout of osr_grid_well_sums; the pointer is kept and read at every
 * evaluation) instead of summing the grid's own layers; NULL restores the
 * grid's own sums. */
osr_status osr_grid_set_well_sums(osr_grid *grid, const double *d_sums);

/* State -> unknowns (InitGuess2, compsim/PetscAUX.cpp:878-964); d_x DEVICE
 * [n_rows]. */
osr_status osr_grid_init_guess(osr_grid *grid, double *d_x, void *stream);

/* Unknowns -> state plus the property sweeps (UpdateAll(x, false),
 * compsim/PetscAUX.cpp:176-498). */
osr_status osr_grid_update_all(osr_grid *grid, const double *d_x, void *stream);

/* Residual rows at the current state (IteratorFunction,
 * compsim/Petsc_Functions.cpp:10-6895) into d_f [n_rows]; d_scale (optional,
 * DEVICE [n_rows]) receives the sum of the absolute values of each row's
 * terms.  sim_time (s) selects the active wells. */
osr_status osr_grid_residual(osr_grid *grid, double *d_f, double *d_scale, double sim_time, void *stream);

/* FormFunction (compsim/PetscAUX.cpp:59-104): osr_grid_update_all then
 * osr_grid_residual. */
osr_status osr_grid_form_function(osr_grid *grid, const double *d_x, double *d_f, double sim_time, void *stream);

/* Residual adjoint with respect to the matrix continuum's per-cell
 * log-permeability theta_c = ln k_c (k_x, k_y, k_z of matrix cell c scaled
 * together): d_gk [cells] = sum_r lambda_r dF_r/d theta_c for a DEVICE
 * vector d_lambda in the residual's row layout, at the grid's current state
 * (call after osr_grid_form_function or osr_grid_update_all at the same
 * unknowns).  The reference has no adjoint; this differentiates its
 * residual (IteratorFunction, compsim/Petsc_Functions.cpp:10-6895) through
 * the matrix faces' interface transmissibilities (IFK_Calc,
 * compsim/Init_Calcs.cpp:21-46) and the convective matrix-fracture shape
 * factor (compsim/Init_Calcs.cpp:970-983).  Well productivity indices are
 * held fixed (their permeability dependence is not differentiated).
 * Deterministic; asynchronous on `stream`. */
osr_status osr_grid_residual_logk_vjp(osr_grid *grid, const double *d_lambda, double *d_gk, double sim_time,
                                      void *stream);

/* ---------------------------------------------------------------------------
 * Jacobian path: the PETSc FormJacobian callback on the device.
 *
 * The matrix is the reference's IteratorJacobian (compsim/Petsc_Functions.cpp:
 * 6898-42073) entry for entry, including its approximate derivatives.  It is
 * returned as a fixed set of values per block row (one cell of one
 * continuum, block rows ordered as osr_grid_refresh_layout orders them):
 *
 *   canonical unknowns of every block (bs = 2N+4 columns):
 *     x_0..x_{N-1}, y_0..y_{N-1}, P, Sw, So, Sg
 *   canonical rows: fugacity 0..N-1, component balances N..2N-2, total
 *     2N-1, water 2N, sum x 2N+1, sum y 2N+2, sum S 2N+3
 *   a one-phase cell's N+3 reference rows and unknowns map onto these; its
 *   unused rows carry a unit entry in an unused column;
 *   eight block slots: this cell, -x, +x, -y, +y, -z, +z neighbours, the
 *     same cell of the other continuum (osr_grid_block_columns);
 *   stored entries, in this order:
 *     fugacity rows x own slot x columns 0..2N          N (2N+1)
 *     rows N..2N-1 x 8 slots x all columns              8 N (2N+4)
 *     water row x 8 slots x {P, Sw}                     16
 *     rows 2N+1..2N+3 x own slot x all columns          3 (2N+4)
 *     eight entries of the total row the reference places in the block after
 *     a neighbour's (its -y / -z face columns counted from the following
 *     block's row offset)                               8
 *
 * vals: DEVICE [ceil(2 cells / 32)][entries][32]: block row b's value e at
 * ((b / 32) entries + e) 32 + b % 32 (entries from osr_grid_jacobian_shape;
 * values of the last chunk beyond the grid are zeros).
 * osr_grid_jacobian_pattern gives every value's
 * reference (global row, global column), -1 for a value the reference's
 * matrix does not hold (unit entries of unused rows, absent neighbours and
 * unknowns); a PETSc adapter passes the pattern to MatSetPreallocationCOO
 * once per row layout and vals to MatSetValuesCOO each call (COO sums
 * duplicates, as the reference's ADD_VALUES does).
 * ------------------------------------------------------------------------- */
osr_status osr_grid_jacobian_shape(osr_grid *grid, int *bs, int *entries, int *overflow);
osr_status osr_grid_block_columns(osr_grid *grid, long *out /* HOST [2 cells][8] */);

/* Reference (row, column) of each value: DEVICE d_row, d_col, same layout
 * as vals.  Depends on the row layout only (osr_grid_refresh_layout). */
osr_status osr_grid_jacobian_pattern(osr_grid *grid, long *d_row, long *d_col, void *stream);

/* The Jacobian at the current state (after osr_grid_update_all or
 * osr_grid_form_function): every cell-medium in any phase state; inactive
 * cell-media (porosity < 1e-10) get a unit diagonal as in the reference.
 * Every value is written (no clearing needed).  Asynchronous on `stream`
 * (the first call on a grid allocates its scratch). */
osr_status osr_grid_jacobian(osr_grid *grid, double sim_time, double *d_vals, void *stream);

/* FormJacobian (compsim/PetscAUX.cpp:106-173): osr_grid_update_all then
 * osr_grid_jacobian. */
osr_status osr_grid_form_jacobian(osr_grid *grid, const double *d_x, double sim_time, double *d_vals,
                                  void *stream);

/* ---------------------------------------------------------------------------
 * Phase appearance after an accepted time step.
 * ------------------------------------------------------------------------- */

/* Saturation pressure of every one-phase cell of one continuum (0 matrix, 1
 * fracture): the bubble pressure of an oil-only cell from its oil pressure,
 * the dew pressure of a gas-only cell from its gas pressure (Bubl_Succ,
 * Dew_Succ, fBubl_Succ, fDew_Succ, compsim/Minor_NR.cpp:491-2015: successive
 * substitution, then a Newton fallback with a dense (N+1)^2 solve).
 * d_psat [cells]: the pressure, -1 where the reference's function returns -1
 * (no convergence in 20 iterations, trivial solution), 0 for two-phase
 * cells.  d_xm [nc][cells] (optional): the incipient phase's composition.
 * DEVICE pointers; asynchronous on `stream`. */
osr_status osr_grid_saturation_pressure(osr_grid *grid, int medium, double *d_psat, double *d_xm, void *stream);

/* Saturation-pressure variants the reference keeps without live call sites
 * (compsim/Do_Cycle.cpp:1576-1605, 1653-1682), on every cell of one
 * continuum (0 matrix, 1 fracture; the reference's functions read the
 * matrix):
 *   kind 0 OSR_SATP_BUBBLE_NR  Bubl_NR (compsim/Minor_NR.cpp:33-266) on oil-only
 *          cells: Newton on the fugacity equalities and the sum of the
 *          incipient gas composition, from Wilson K-values at the oil pressure;
 *   kind 1 OSR_SATP_DEW_NR     Dew_NR (compsim/Minor_NR.cpp:268-489) on gas-only
 *          cells, from the gas pressure;
 *   kind 2 OSR_SATP_LOWER_DEW  LowerDew_Succ (compsim/Minor_NR.cpp:2017-2136)
 *          on gas-only cells: the lower dew point by substitution, 1e100 for a
 *          trivial solution.
 * d_psat [cells] the pressure (0 for cells of the other labels); d_xm
 * [nc][cells] (optional) the incipient composition of the last iterate;
 * d_status [cells] (optional) osr_cell_status: OSR_CELL_MAXIT where the
 * Newton forms did not stop within 100 steps (the reference iterates without
 * a cap), OSR_CELL_NAN for a non-finite pressure; d_iters [cells] (optional)
 * the steps taken.  DEVICE pointers; asynchronous on `stream`. */
enum { OSR_SATP_BUBBLE_NR = 0, OSR_SATP_DEW_NR = 1, OSR_SATP_LOWER_DEW = 2 };
osr_status osr_grid_saturation_pressure_nr(osr_grid *grid, int medium, int kind, double *d_psat, double *d_xm,
                                           int *d_status, int *d_iters, void *stream);

/* critTest (compsim/Minor_NR.cpp:2138-2308): the successive-substitution
 * stability test of every one-phase cell of one continuum at its oil
 * pressure.  An oil-only cell whose flash gives L = 0 becomes gas-only (its
 * oil composition and saturation move to the gas); a gas-only cell whose
 * flash gives L = 1 becomes oil-only.  d_L [cells] (optional): the final L
 * (-1 for two-phase cells); d_changed (optional, one int the caller zeroes):
 * incremented by the number of relabelled cells.  A relabelled cell changes
 * the row layout: follow with osr_grid_refresh_layout.  DEVICE pointers;
 * asynchronous on `stream`. */
osr_status osr_grid_crit_test(osr_grid *grid, int medium, double *d_L, int *d_changed, void *stream);

/* PhaseCtrl and fPhaseCtrl (compsim/Do_Cycle.cpp:1558-1721) on the current
 * state: phase appearance at 0.95 of the saturation pressure with a new-phase
 * saturation of 1e-3 and the incipient composition, phase disappearance at
 * zero saturation, saturations renormalised.  Changes labels, saturations
 * and compositions; the row layout follows with osr_grid_refresh_layout. */
osr_status osr_grid_phase_ctrl(osr_grid *grid, void *stream);

/* UpdateAll(x, true) after an accepted Newton solve (compsim/PetscAUX.cpp:
 * 176-498, UpdateDependencies(true) :500-545): unpack x, PhaseCtrl and
 * fPhaseCtrl, PCoeff and the row layout, then the property sweeps.
 * Synchronises `stream` (the new row count and PCoeff come back to the host). */
osr_status osr_grid_update_all_full(osr_grid *grid, const double *d_x, void *stream);

/* ---------------------------------------------------------------------------
 * Linear solve of the Newton system (replaces the KSPSolve inside SNESSolve
 * of SolveNonLinear, compsim/PetscAUX.cpp:631-646, 672-698: SNESKSPONLY,
 * KSPBCGS, PCVPBJACOBI over the PJac block sizes, KSPSetTolerances with the
 * deck's RELTOL / ABSTOL / DIVTOL / MAXITERS, compsim/Data_Input.cpp:232-266).
 * The matrix is the compact Jacobian of osr_grid_jacobian for the grid's
 * current row layout; vectors are DEVICE arrays of the layout's row count.
 * ------------------------------------------------------------------------- */
typedef struct {
    double rtol;      /* RELTOL, default 1e-18 */
    double atol;      /* ABSTOL, default 1e-50 */
    double dtol;      /* DIVTOL, default 1e3 */
    int max_it;       /* MAXITERS, default 5000 */
    int check_every;  /* iterations enqueued between host status reads (8) */
} osr_ksp_opts;

typedef struct {
    int reason;       /* PETSc KSPConvergedReason: 2 CONVERGED_RTOL, 3 CONVERGED_ATOL,
                         -3 DIVERGED_ITS, -4 DIVERGED_DTOL, -5 DIVERGED_BREAKDOWN,
                         -9 DIVERGED_NANORINF, -11 DIVERGED_PC_FAILED (zero pivot) */
    int its;          /* iterations taken */
    double rnorm0;    /* |B b|_2, the initial preconditioned residual */
    double rnorm;     /* final preconditioned residual 2-norm */
} osr_ksp_info;

/* The reference's defaults (compsim/Data_Input.cpp:232-266). */
void osr_ksp_default_opts(osr_ksp_opts *opts);

/* y = J x (MatMult) on the compact Jacobian d_vals.  Asynchronous. */
osr_status osr_grid_jacobian_apply(osr_grid *grid, const double *d_vals, const double *d_x, double *d_y,
                                   void *stream);

/* y = J^T lambda (MatMultTranspose) on the compact Jacobian d_vals: the
 * vector-Jacobian product of the residual in the unknowns at the state the
 * Jacobian was formed at (the step an adjoint of the Newton system takes).
 * Every stored value adds value * lambda[row] into y[column] of its reference
 * (row, column); values that are exactly zero are skipped.  Atomic additions:
 * the last bits may differ between runs.  DEVICE vectors of the layout's row
 * count; asynchronous. */
osr_status osr_grid_jacobian_apply_transpose(osr_grid *grid, const double *d_vals, const double *d_lambda,
                                            double *d_y, void *stream);

/* Solve J d_sol = d_rhs from a zero initial guess with left-preconditioned
 * BiCGStab and the inverse diagonal blocks of J (one block per cell-medium)
 * as preconditioner, PETSc's KSPBCGS + PCVPBJACOBI.  opts may be null (the
 * defaults).  Synchronises `stream` every opts->check_every iterations; the
 * outcome is in info (may be null): a solve that does not converge returns
 * OSR_OK with a negative info->reason, as KSPSolve does. */
osr_status osr_grid_ksp_solve(osr_grid *grid, const double *d_vals, const double *d_rhs, double *d_sol,
                              const osr_ksp_opts *opts, osr_ksp_info *info, void *stream);

/* Solve J^T d_sol = d_rhs (the adjoint system of the Newton step) from a zero
 * initial guess: the same left-preconditioned BiCGStab with J^T in the
 * products (the transposed product of osr_grid_jacobian_apply_transpose)
 * and the transposed inverse diagonal blocks as preconditioner.  Options,
 * outcome and synchronisation as osr_grid_ksp_solve. */
osr_status osr_grid_ksp_solve_transpose(osr_grid *grid, const double *d_vals, const double *d_rhs, double *d_sol,
                                        const osr_ksp_opts *opts, osr_ksp_info *info, void *stream);

/* ---------------------------------------------------------------------------
 * Distributed linear solve over z-slabs (the multi-rank KSPSolve of the
 * reference: PETSc's KSPBCGS + PCVPBJACOBI over CreateAllocationTable's row
 * ownership, compsim/PetscAUX.cpp:1081-1099, with VecDot / VecNorm summed over
 * the ranks).  Each rank holds one slab grid (its owned layers plus one ghost
 * layer towards each neighbour) and the slab's compact Jacobian.  The
 * iteration above is split at its dot products into stages: every stage's
 * partial sums over the slab's OWNED rows land in d_dots, which the caller
 * sums over the ranks (an all-reduce on `stream`) before the next stage, and
 * the caller refills the ghost rows of d_p (after stage 1) and d_s (after
 * stage 3) from the neighbouring ranks.  Protocol:
 *   osr_dksp_begin  (dots[0]: sum)   osr_dksp_stage 0
 *   per iteration:  stage 1 (ghosts of p), 2 (dots[0]: sum), 3 (ghosts of s),
 *                   4 (dots[0..2]: sum), 5 (dots[0..1]: sum), 6
 *   osr_dksp_info every few iterations; stop once info.reason != 0.
 * Every rank takes the same scalar steps from the same sums, so all ranks
 * stop at the same iteration.  With one rank owning every row the stages
 * perform the single-grid solve's arithmetic exactly.  The handle shares the
 * grid's solve workspace: a distributed solve and osr_grid_ksp_solve on the
 * same grid do not interleave.
 * ------------------------------------------------------------------------- */
typedef struct osr_dksp osr_dksp;
osr_status osr_dksp_create(osr_grid *grid, osr_dksp **out);
void osr_dksp_destroy(osr_dksp *dksp);
/* Start solving J x = b from x = 0.  owned[4]: the owned block rows
 * [owned[0], owned[1]) of the matrix continuum and [owned[2], owned[3]) of
 * the fracture continuum (cell-medium indices, fracture from `cells`).
 * d_x, d_p, d_s: the caller's DEVICE vectors of the grid's row count (the
 * solution, and the two search vectors whose ghost rows the caller fills);
 * d_dots: at least 3 doubles.  Asynchronous on `stream`. */
osr_status osr_dksp_begin(osr_dksp *dksp, const double *d_vals, const double *d_b, double *d_x, double *d_p,
                          double *d_s, const long *owned, const osr_ksp_opts *opts, double *d_dots, void *stream);
/* One stage (0..6; see above).  Asynchronous on `stream`. */
osr_status osr_dksp_stage(osr_dksp *dksp, int stage, void *stream);
/* The solve's state (reason 0 while running).  Synchronises `stream`. */
osr_status osr_dksp_info(osr_dksp *dksp, osr_ksp_info *info, void *stream);

/* ---------------------------------------------------------------------------
 * Time stepping: one osr_sim_step is one pass of the reference's main loop
 * (compsim/PrimeSim.cpp:93-104).  SolveNonLinear (compsim/PetscAUX.cpp:
 * 566-731): the unknowns of the current state, F and J there, one linear
 * solve (osr_grid_ksp_solve), x - dx; accepted when the solve converged and
 * |dx|_1 / rows <= 1e-2 (TOLMAIN), then UpdateAll(x, true) and CreateBackups.
 * TimeStepCtrl (compsim/Do_Time_Step.cpp:391-470): the time advances by Dt,
 * Dt x 1.03 after every 5 accepted steps, clamped to [1e-10 s, max_dt] and
 * cut to the next marker; a rejected pass divides Dt by 1.5 and restores the
 * backed-up state (RestoreBackups + PJac, :354-389).
 * ------------------------------------------------------------------------- */
typedef struct osr_sim osr_sim;

typedef struct {
    double sim_time;  /* simulation time after the pass (s) */
    double dt;        /* Dt of the next pass (s) */
    int accepted;     /* the pass's solve was accepted */
    int finished;     /* the last time marker was reached (the reference's loop ends) */
    int ksp_reason;   /* osr_ksp_info.reason of the pass's linear solve */
    int ksp_its;
    double vnorm;     /* |dx|_1 / rows */
    long rows;        /* rows of the pass's system */
} osr_step_info;

/* A run on `grid` from its current state (set by the caller): markers are
 * the ascending time markers (s) -- every well's start and end time and the
 * total time, merged as ManageTSMarker does (compsim/Init_Calcs.cpp:
 * 1133-1157) -- dt the first Dt, max_dt the deck's DTMAX.  Runs the property
 * sweeps and the row layout of the current state and takes the first backup
 * (compsim/PrimeSim.cpp:85-86).  The grid must outlive the run. */
osr_status osr_sim_create(osr_grid *grid, const double *markers, int n_markers, double dt, double max_dt,
                          osr_sim **sim);

/* One pass (see above).  opts: the linear solve's tolerances (null: the
 * reference's defaults).  Synchronises `stream`.  Returns
 * OSR_ERR_UNSUPPORTED when Dt falls below 1e-10 s (the reference stops with
 * "MINDT was hit"); after the last marker a call does nothing and reports
 * finished. */
osr_status osr_sim_step(osr_sim *sim, const osr_ksp_opts *opts, osr_step_info *info, void *stream);

/* Whether osr_sim_step runs a pass as one CUDA graph (default on): InitGuess2,
 * FormFunction, FormJacobian, the linear solve, x - dx, the acceptance test
 * and, by a device-side if / else, UpdateAll(x, true) + CreateBackups or
 * RestoreBackups + PJac; TimeStepCtrl follows on the host.  The graph reads
 * the pass's Dt, time and PCoeff from device memory, so one capture serves
 * every pass until the row count changes, and it gives exactly the direct
 * launches' results.  Off: direct launches. */
osr_status osr_sim_set_graph(osr_sim *sim, int on);
/* Passes run through the step graph so far. */
osr_status osr_sim_graph_launches(osr_sim *sim, long *launches);
/* The current step graph: 0 none, 1 linearisation and solve only (the
 * acceptance and UpdateAll by direct launches), 2 the whole pass. */
osr_status osr_sim_graph_form(osr_sim *sim, int *form);

/* Current simulation time and Dt (either may be null). */
osr_status osr_sim_time(osr_sim *sim, double *sim_time, double *dt);

/* Index of the next time marker (the reference's TSMCtrl, written to its
 * restart file). */
osr_status osr_sim_marker_index(osr_sim *sim, int *tsm_ctrl);

/* Continue a run from a restart file (ReadRST, compsim/Do_Time_Step.cpp:
 * 236-294): simulation time, Dt and marker index as read; the grid's
 * current state (set from the file) becomes the backup. */
osr_status osr_sim_restart(osr_sim *sim, double sim_time, double dt, int tsm_ctrl);

/* The reference's restart file for a C++ host (WriteRST / ReadRST,
 * compsim/Do_Time_Step.cpp:179-294): both continua's phase pressures with the
 * one-cell halo (written as zeros), per cell the saturations, the liquid and
 * vapour compositions and the label, then simTime, Dt, TSMCtrl and SMethQ
 * (the main loop's cumulative producer methane, which the device run does
 * not track: the caller passes it).  Reading restores the state, then
 * PhaseCtrl, the row layout, the property sweeps and the run's time, Dt and
 * marker (ReadRST + UpdateDependencies(true) + CreateBackups,
 * compsim/PrimeSim.cpp:84-86); a file of another grid or component count is
 * OSR_ERR_ARG.  HOST paths; synchronous. */
osr_status osr_sim_write_restart(osr_sim *sim, const char *path, double smethq);
osr_status osr_sim_read_restart(osr_sim *sim, const char *path, double *smethq);

/* The reference's state listing (PrintAll, compsim/ViewAssist.Cpp:39-88)
 * appended to `path`: 80 dashes, the time in hours (%g on the stream's first
 * call, first_call != 0, then %.20g), the header, then per matrix and per
 * fracture cell (z outermost, x fastest) the indices, oil pressure,
 * saturations and both phase compositions at 20 significant digits.
 * Synchronous. */
osr_status osr_grid_write_listing(osr_grid *grid, const char *path, double sim_time, int first_call);

osr_status osr_sim_destroy(osr_sim *sim);

/* Measured FP64 FMA-pipe throughput of the current device in TFLOP/s (an FMA
 * counts 2): a dependent-FMA microbenchmark, best of 5 launches.  The
 * denominator of the flash kernel's roofline.  No reference counterpart. */
osr_status osr_probe_fp64_peak(double *tflops, void *stream);

/* The flash kernels' branch-free quotient and reciprocal on n operand pairs
 * (DEVICE pointers): d_q[i] = a_i / b_i, d_r[i] = 1 / b_i as the kernels
 * compute them, and d_ok[i] = 1 where the operands are inside the range the
 * kernels accept without their IEEE fallback.  A test hook for the
 * quotients' accuracy against IEEE division; no reference counterpart. */
osr_status osr_probe_quotients(const double *d_a, const double *d_b, long n, double *d_q, double *d_r,
                               signed char *d_ok, void *stream);

/* Error reporting. */
const char *osr_status_string(osr_status s);
int osr_last_cuda_error(void);

/* Blocks the library has taken from its stream-ordered device pools since
 * the process started (every allocating entry point counts here; the
 * no-allocation entry point never does).  A diagnostic; no reference
 * counterpart. */
long osr_pool_alloc_count(void);
int osr_version(void);

#ifdef __cplusplus
}
#endif
#endif
