/*
 * trench_b200 -- C ABI of the B200 (sm_100a) charging-step backend.
 *
 * Every entry point returns an int status (TB_OK = 0, >0 a TB_ERR_* code) and
 * never throws or aborts; tb_last_error() gives the message of the last failure
 * on a context (or of a failed tb_create when ctx is NULL).  Array pointers named
 * d_* are DEVICE pointers on the context's device (any allocator: torch, cudaMalloc);
 * h_* are host pointers.  `stream` is a cudaStream_t (NULL = default stream).
 * One context serves one trench case (fixed grid and vacuum mask); a context is
 * not thread-safe, distinct contexts are independent.
 *
 * Grids are (nx, ny) in C order: cell (ix, iy) is element ix*ny + iy, x periodic,
 * iy = 0 at the substrate -- the layout of the reference's NumPy arrays.
 */
#ifndef TRENCH_B200_H
#define TRENCH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TB_OK 0
#define TB_ERR_ARG 1          /* invalid argument or shape (Python: ValueError) */
#define TB_ERR_CUDA 2         /* CUDA runtime failure (Python: RuntimeError) */
#define TB_ERR_DEVICE 3       /* device index not available (Python: RuntimeError) */
#define TB_ERR_KERNEL 4       /* a kernel reported a failed internal check */
#define TB_ERR_CONVERGENCE 5  /* iterative solve did not reach its tolerance */

#define TB_PRECISION_F64 0    /* reference-exact FP64 arithmetic, fields from global memory */
#define TB_PRECISION_F32 1    /* FP32, cell + offset positions, fields staged in shared memory */

typedef struct tb_ctx tb_ctx;

/* Arguments of one tracer launch.  Replaces the argument list of the reference
 * kernel `trace_particles` (trench_trace.cu:70-77) and of the host call
 * CudaTracer.__call__ (trench_cuda.py:41).  Unused optional pointers are NULL. */
typedef struct {
    int64_t n;                       /* particles */
    double *d_x, *d_y, *d_vx, *d_vy; /* SoA state, metres and m/s; updated in place when
                                        write_state != 0 */
    const double *d_qm;              /* charge/mass, C/kg */
    const int8_t *d_spc;             /* species: 0 ion, 1 electron */
    /* FP64 fields (nx*ny each).  Precision F64 reads them directly; precision F32
       reads the packed copy made by tb_set_fields and ignores these. */
    const double *d_ex, *d_ey;
    const double *d_phi, *d_wface;   /* wall barrier (wall_model="barrier"); NULL = absorb */
    int max_steps;                   /* per-particle step cap (total over launches) */
    int step_budget;                 /* steps this launch (<= max_steps); chunked runs */
    double cfl;
    int tapered;                     /* corner crossing + first-face deposit (trench_charging_2d.py:554) */
    /* circuit_rf in-flight clock; n_phase = 0 disables.  Precision F32 reads the
       basis fields packed by tb_set_rf_fields instead of these three. */
    const double *d_rf_ex, *d_rf_ey, *d_rf_phi; /* (2, nx, ny) */
    const double *d_wave;            /* (n_phase, 2) */
    int n_phase;
    double period, dt_max, bound_vs, bound_vm;
    double *d_clock;                 /* (n, 2): clock, elapsed; in/out */
    /* trajectory record (F64 only) */
    int record;
    double *d_endpoints;             /* (n, 2) in/out */
    const int32_t *d_slots;          /* (n) path slot or -1 */
    double *d_paths;                 /* (slots, path_stride, 2) */
    int32_t *d_path_len;             /* (slots) in/out */
    int path_stride;
    /* outputs */
    int32_t *d_counts;               /* (2, nx, ny) hit histogram per species, accumulated */
    int64_t *d_totals;               /* [8] escaped ions, escaped electrons, lost, particle-steps,
                                        absorbed ions, absorbed electrons, -, -; accumulated */
    int8_t *d_status;                /* (n) 1 absorbed, 2 escaped, 3 live; in/out, required */
    int32_t *d_hit;                  /* (n) absorbing cell or -1; optional */
    int32_t *d_steps;                /* (n) steps taken; in/out, required */
    int write_state;                 /* write final x, y, vx, vy back */
} tb_trace_args;

int tb_version(void);

/* Create a context on `device` for an (nx, ny) grid with cell size dx (m) and
 * vacuum mask h_vac (1 = vacuum).  Replaces CudaTracer.__init__ (trench_cuda.py:24-39). */
int tb_create(tb_ctx **out, int device, int nx, int ny, double dx, const uint8_t *h_vac);
int tb_destroy(tb_ctx *ctx);
const char *tb_last_error(const tb_ctx *ctx);
/* Device name and SM count of the context's GPU. */
int tb_device_info(const tb_ctx *ctx, char *name, int name_len, int *num_sms);

/* Pack FP64 fields into the FP32 shared-memory layout used by precision F32:
 * E*vac scaled to cell units, the vacuum flag, and the per-face wall barrier
 * (d_phi/d_wface may be NULL for the absorb model).  vscale (m/s) is the
 * velocity unit of the FP32 state.  The tracer of trench_cuda.py:61,80 copies
 * these arrays to the GPU on every call; here they stay resident. */
int tb_set_fields(tb_ctx *ctx, const double *d_ex, const double *d_ey, const double *d_phi,
                  const double *d_wface, double vscale, void *stream);

/* Pack the circuit_rf unit-voltage basis fields ((2, nx, ny) Ex, Ey and potential:
 * substrate then mask electrode) and the waveform ((n_phase, 2) voltage deltas over
 * one period) for precision F32 with the RF clock: the fields as one float4 per cell,
 * the per-face barrier of each basis potential, in the units of the last
 * tb_set_fields (call it again after a tb_set_fields with another vscale), and the
 * waveform as one float4 per table interval.  The basis and waveform are fixed for a
 * case, so one call serves every batch; tb_trace then requires args->d_wave and
 * n_phase to be the ones given here.  A later call with a longer waveform moves the
 * table: capture CUDA graphs of traces after the last call.  Replaces the copies of rf_ex/rf_ey/rf_phi/wave
 * in CudaTracer.__call__ (trench_cuda.py:63-70). */
int tb_set_rf_fields(tb_ctx *ctx, const double *d_rf_ex, const double *d_rf_ey, const double *d_rf_phi,
                     const double *d_wface, const double *d_wave, int n_phase, void *stream);

/* Trace particles until absorbed, escaped or max_steps; deposit hits into
 * d_counts with integer atomics.  Replaces the chunk loop, kernel launch and host
 * bincount of CudaTracer._trace (trench_cuda.py:100-122) and the kernel
 * trace_particles (trench_trace.cu:70-193). */
int tb_trace(tb_ctx *ctx, const tb_trace_args *args, int precision, void *stream);

/* Launch shape of the FP32 tracer on this context: CTA size 128, 256, 512, 768 or 1024
 * threads and 1 or 2 CTAs per SM (2 only where two shared-memory fields fit on an SM),
 * or threads = 0: chosen per launch from the batch size (the default).  The launch uses
 * ceil(n / threads) CTAs up to SMs x CTAs per SM, so small CTAs spread a small batch
 * over more SMs; the default takes the largest CTA that still gives every SM one (1024
 * threads for batches of SMs x 768 particles and more, 128 at the least).  Chosen by the
 * autotuner (ChargingCase.autotune_tracer). */
int tb_set_tuning(tb_ctx *ctx, int threads, int ctas_per_sm);
/* Order in which the FP32 tracer's lanes claim particles: 0 in index order
 * (default), 1 from the last index down, 2 learned: every electron first, then the
 * ions longest predicted first, the prediction being the mean step count of the ion's
 * bin (starting column band, direction band) in the previous trace on this context
 * (three small kernels before the trace write claim records in that order, two after
 * it learn the bins; circuit_rf launches claim in index order).  Results do not depend
 * on the order; the time does, because a launch ends with the particles still in
 * flight when the queue runs dry.  The learned order's buffers are allocated by
 * tb_reserve_claim_order or by the first trace that uses it outside a stream capture; a
 * trace captured before either claims in index order.  Chosen by the autotuner. */
int tb_set_claim_order(tb_ctx *ctx, int order);
/* Allocates the learned claim order's buffers for batches of up to n particles (about
 * 34 bytes per particle), so that a CUDA graph captured afterwards uses the order.  Not
 * during a stream capture. */
int tb_reserve_claim_order(tb_ctx *ctx, long long n);

/* Synchronise `stream`, then read and clear the context's device-side check flag:
 * TB_ERR_KERNEL if a kernel recorded a failed bound (a deposit cell outside the
 * grid, a bulk copy that did not complete in its bounded wait).  After
 * TB_ERR_KERNEL the batch's counts, totals, status and step counts are partial (a
 * CTA whose field copy timed out returned without tracing its particles): discard
 * them and trace the batch again. */
int tb_check(tb_ctx *ctx, void *stream);

/* ---- Poisson: multigrid-preconditioned CG ------------------------------------
 * Operator L = -dx^2 A, the SPD form of the reference's 5-point matrix
 * (trench_charging_2d.py:252-294): per cell the diagonal d > 0 and the
 * couplings kE (to ix+1, periodic) and kN (to iy+1) >= 0, host arrays of nx*ny.
 * Cells with h_fixed != 0 are Dirichlet zero.  Replaces the SuperLU factorisation
 * and solve of make_solver / setup_fields (trench_charging_2d.py:297-309, 378-392). */
int tb_poisson_setup(tb_ctx *ctx, const double *h_diag, const double *h_ke, const double *h_kn,
                     const uint8_t *h_fixed, int max_rhs);
/* V-cycle schedule: smoothing sweeps before/after the coarse correction and on the
 * coarsest level (defaults 1, 1, 16).  Chosen by the autotuner (FieldSolver.autotune). */
int tb_poisson_schedule(tb_ctx *ctx, int pre, int post, int coarse_sweeps);
/* Number of multigrid levels built by tb_poisson_setup (0 before setup). */
int tb_poisson_levels(const tb_ctx *ctx);
/* Solve L x = b for nrhs right-hand sides, d_b and d_x (nrhs, nx*ny) FP64; d_x is
 * the initial guess on entry.  b must be zero on fixed cells.  Stops when every
 * relative residual |b - L x| / |b| <= rtol, after at most max_outer FP64
 * refinement steps of `inner` FP32 PCG iterations each.  Synchronises `stream`
 * once per refinement step.  TB_ERR_CONVERGENCE if rtol is not reached. */
int tb_poisson_solve(tb_ctx *ctx, int nrhs, const double *d_b, double *d_x, double rtol, int max_outer,
                     int inner, int *iters, double *h_resid, void *stream);

/* ---- Per-batch charge and field update ------------------------------------------
 * The state is the charge density on the m surface cells (charge is only ever
 * deposited there); the potential is phi = external + G rho_s with G the surface
 * Green's operator built once with tb_poisson_solve.  Together the two calls
 * replace the body of the reference batch loop after the trace
 * (trench_charging_2d.py:1239-1285). */
#define TB_SFLAG_COND 1u     /* surface cell is a conductor cell */
#define TB_SFLAG_REGION 2u   /* counted in the leakage current monitor */
#define TB_SFLAG_BOTTOM 4u   /* bottom row (floor_t-1) inside the bottom opening */

typedef struct {
    int m;                           /* surface cells */
    const int32_t *d_surf;           /* (m) flat cell index */
    const uint8_t *d_sflag;          /* (m) TB_SFLAG_* bits */
    double *d_rho_s;                 /* (m) charge density, C/m^3 (state) */
    double *d_rho_prev;              /* (m) scratch */
    double *d_work;                  /* (2m) scratch */
    const double *d_leak_M;          /* (m, m) implicit leakage operator, NULL = no leakage */
    const double *d_leak_h;          /* (m) dt G phi_ext on surface cells, or NULL */
    const double *d_g_s;             /* (m) floating-conductor response at surface cells, or NULL */
    int c_slot;                      /* surface index holding the floating conductor's charge, or -1 */
    int floating, driven;
    double q_macro, dx, C_cond, Te, dt_batch, leak_norm, bottom_norm, n_per_batch;
    int n_rows;                      /* cells whose potential is needed (vacuum + surface) */
    const int32_t *d_rows;           /* (n_rows) flat cell index */
    const float *d_green;            /* (n_rows, m) FP32 Green's operator, or NULL */
    const double *d_green64;         /* (n_rows, m) FP64 Green's operator, or NULL */
    const double *d_ext;             /* (nx*ny) external potential */
    double *d_phi;                   /* (nx*ny) potential; rows are rewritten each batch */
    double *d_ex, *d_ey;             /* (nx*ny) FP64 field, or NULL */
    const double *d_wface;           /* (nx*ny) wall barrier weight, NULL = absorb model */
    double v_sub, v_top;             /* ghost-cell voltages of the field (trench_charging_2d.py:446-447) */
    int top_dirichlet;
    double vscale;                   /* velocity unit of the FP32 tracer state, m/s */
    double *d_hist;                  /* (max_batches, hist_cols): ratio_i, ratio_e, esc_e, lost, leak,
                                        particle-steps, probe potentials... */
    int hist_cols, max_batches;
    int n_probes;
    const int32_t *d_probes;         /* (n_probes) flat cell index */
    int32_t *d_batch;                /* device batch counter (start at -1) */
    const int32_t *d_counts;         /* (2, nx*ny) tracer counts of this batch */
    const int64_t *d_totals;         /* tracer totals of this batch */
} tb_step_desc;

/* Deposit, leakage, conductor step and history scalars (one batch). */
int tb_step_charge(tb_ctx *ctx, const tb_step_desc *desc, void *stream);
/* Potential on the needed cells, FP64 field, packed FP32 tracer field (as
 * tb_set_fields) and probe history. */
int tb_step_potential(tb_ctx *ctx, const tb_step_desc *desc, void *stream);
/* Charge monitors of the history (trench_charging_2d.py:871-874, 1281-1285): for each
 * of n_monitors, dx^2 sum_s weights[r][s] rho_s (or |rho_s| where absolute[r] != 0)
 * over the m surface slots, written to row *d_batch of d_out (max_batches, n_monitors).
 * Call after tb_step_charge. */
int tb_step_monitors(tb_ctx *ctx, const tb_step_desc *desc, const double *d_weights, const uint8_t *d_absolute,
                     int n_monitors, double *d_out, void *stream);
/* The per-batch state before a trace in one launch (the reference sets it per call,
 * trench_cuda.py:73-74): d_status[0..n) = 3 (untraced), d_steps[0..n) = 0,
 * d_counts[0..n_counts) = 0 and d_totals[0..n_totals) = 0 (n_totals <= 64). */
int tb_batch_reset(tb_ctx *ctx, int8_t *d_status, int32_t *d_steps, long long n, int32_t *d_counts,
                   long long n_counts, unsigned long long *d_totals, int n_totals, void *stream);

/* ---- Device-side injection -------------------------------------------------------
 * Samples n_species ions (indices [0, n)) then n_species electrons ([n, 2n)) into the
 * particle arrays, restating the reference's `inject` (trench_charging_2d.py:458-489)
 * on the GPU.  Random numbers: Philox4x32-10, counter (i, batch) and key seed, so the
 * draws do not depend on the launch.  Ion energy (eV) and polar angle (rad) come from
 * histogram tables (bin edges and cumulative weights, n + 1 entries each, sampled
 * linearly within a bin); n_energy = 0 uses ion_energy_eV, n_angle = 0 a lateral
 * thermal velocity N(0, ion_lateral_sigma).  No counterpart in the reference, which
 * samples on the host with NumPy. */
typedef struct {
    int64_t n_species;
    uint64_t seed, batch;
    double *d_x, *d_y, *d_vx, *d_vy, *d_qm;
    int8_t *d_spc;
    double lx, y0;                   /* domain width and injection height, metres */
    double qm_ion, qm_electron;      /* C/kg */
    double ion_mass, e_charge;       /* kg, C */
    double electron_sigma;           /* sqrt(Te e / m_e), m/s */
    double ion_energy_eV, ion_lateral_sigma;
    const double *d_energy_edges, *d_energy_cdf;
    int n_energy;                    /* bins of the energy table, 0 = fixed energy */
    const double *d_angle_edges, *d_angle_cdf;
    int n_angle;                     /* bins of the angle table, 0 = lateral thermal */
    int angle_random_sign;           /* draw the sign of the angle with probability 1/2 */
    const int32_t *d_counter;        /* optional device batch counter: the Philox batch word is
                                        batch + *d_counter + 1 (lets a CUDA graph replay a new batch) */
    uint16_t *d_bin_e, *d_bin_a;     /* optional (n_species): table bin of each ion's energy / angle
                                        (0 when that quantity has no table); the adjoint's histories */
    double *d_clock;                 /* optional circuit_rf clock (2 n_species, 2): launch time, 0 */
    double period;                   /* RF period (s): each species' launch times are stratified over
                                        one period, particle k of a species in stratum k
                                        (trench_rf.py:14-18; the shuffle there only decorrelates
                                        strata from draws made in sequence, which counter-based
                                        draws are not) */
} tb_inject_args;

int tb_inject(tb_ctx *ctx, const tb_inject_args *args, void *stream);
/* The raw Philox4x32-10 stream: 4 words per index i < n for counter (i, batch) and
 * key seed, into d_out (4n words).  For checking the generator. */
int tb_philox_fill(tb_ctx *ctx, unsigned long long seed, unsigned long long batch, int n, uint32_t *d_out,
                   void *stream);

/* ---- Case packs: many trench cases in one persistent FP32 launch -----------------
 * A pack groups contexts of one device (different grids allowed).  tb_pack_set_args
 * takes one tb_trace_args per case (FP32 rules of tb_trace, circuit_rf cases
 * included; the cases' fields, and RF cases' basis, must have been packed) and is
 * synchronous; tb_pack_trace launches one persistent kernel
 * whose CTAs pick the case with the most unclaimed particles, stage its field in
 * shared memory and trace from its queue, so cases of uneven size share all SMs.
 * reset != 0 first sets status = live, steps = 0 and zeroes counts and totals of every
 * case.  No counterpart in the reference, which runs cases one after another. */
typedef struct tb_pack tb_pack;
int tb_pack_create(tb_pack **out, int n_cases, tb_ctx *const *ctxs);
int tb_pack_destroy(tb_pack *pack);
const char *tb_pack_last_error(const tb_pack *pack);
int tb_pack_set_args(tb_pack *pack, const tb_trace_args *args);
int tb_pack_trace(tb_pack *pack, int reset, void *stream);
/* The per-batch update (tb_step_charge then tb_step_potential) of every case of the
 * pack in one launch per stage -- the charge update of all cases (one 8-CTA cluster
 * per case; a case with more than 1024 surface slots runs its own), then the Green's
 * product of all cases, then their fields -- instead of 3 launches per case.
 * tb_pack_set_steps takes one step descriptor per case, in the pack's case order, and
 * is synchronous; the results equal tb_step_charge + tb_step_potential per case.  No
 * counterpart in the reference. */
int tb_pack_set_steps(tb_pack *pack, const tb_step_desc *descs);
int tb_pack_step(tb_pack *pack, void *stream);
/* Synchronise `stream`, then read and clear the pack's device check flag; after
 * TB_ERR_KERNEL the batch's results are partial, as for tb_check. */
int tb_pack_check(tb_pack *pack, void *stream);

/* ---- No-allocation FP32 tracer ---------------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc -- a
 * host application whose memory pool owns all device memory, or a caller that must
 * not let cudaMalloc/cudaFree synchronise the device -- this entry point allocates
 * nothing and needs no context: the tracer's scratch (packed FP32 field, wall
 * barrier, work-queue counter, check flag) lives in a static device array of about
 * 2.5 MiB that every GPU loading the library holds until the process exits.  It
 * traces like tb_trace with TB_PRECISION_F32 on the current device; the caller
 * passes the device vacuum mask d_vac (nx*ny bytes, 1 = vacuum), the FP64 fields
 * in args->d_ex/d_ey (and d_phi/d_wface for the barrier model) and every input and
 * output array.  Grids above TB_NOALLOC_MAX_CELLS cells are rejected (TB_ERR_ARG).
 * args->d_totals[6] receives the device check flag (0 = every bound held; a raised
 * flag means the batch's results are partial and must be traced again, as after
 * tb_check's TB_ERR_KERNEL); with n = 0 it is set to 0.  Every call looks up the
 * array's device address and sets the kernel's shared-memory attribute (host-side
 * calls that allocate nothing), so a call after a device reset finds the reloaded
 * module; the first call on a device also loads the module, so make it before any
 * stream capture.  All calls share the
 * one array, so calls that overlap on the GPU (other streams, other host threads)
 * race: serialise them.  Errors are read with tb_last_error(NULL). */
#define TB_NOALLOC_MAX_CELLS 65536
int tb_trace_f32_noalloc(int nx, int ny, double dx, const uint8_t *d_vac, const tb_trace_args *args,
                         double vscale, void *stream);

/* ---- Adjoint of the charging loop -----------------------------------------------
 * No counterpart in the reference, which has no gradient.  The gradient of a
 * charging objective with respect to the ion energy/angle histogram weights and the
 * surface charge is taken by likelihood-ratio reweighting of the traced histories:
 * per batch b the absorbed ions are tallied by (table bin, surface slot), so that a
 * change of the bin probabilities by factors rE[k], rA[l] changes the expected ion
 * deposit on slot s to
 *     ci_b[s](r) = Ni_b[s] + sum_k (rE[k] - 1) TE_b[k][s] + sum_l (rA[l] - 1) TA_b[l][s]
 * (Ni_b = the traced count; first order in r - 1, exact at r = 1).  The charge
 * update of tb_step_charge then runs over these deposits -- the surrogate recurrence,
 * traced histories held fixed -- and its adjoint is swept backwards, optionally with
 * the deposits' measured response to the charge state (field feedback) added. */

/* Tally one traced batch.  Ions are particles [0, n_species), electrons
 * [n_species, 2 n_species).  An absorbed particle (status 1) on cell c adds 1 in
 * column d_slot[c] of the table, (n_energy + n_angle + 2, m) int32, accumulated:
 * an ion to rows bin_e, n_energy + bin_a and n_energy + n_angle (all ions), an
 * electron to row n_energy + n_angle + 1.  A bin index out of range, or an absorbed
 * particle off the surface, raises the context's device check flag (tb_check). */
typedef struct {
    int64_t n_species;
    const int8_t *d_status;          /* (2 n_species) */
    const int32_t *d_hit;            /* (2 n_species) absorbing cell */
    const uint16_t *d_bin_e, *d_bin_a; /* (n_species) */
    const int32_t *d_slot;           /* (nx*ny) surface slot of each cell or -1 */
    int m, n_energy, n_angle;
    int32_t *d_table;
} tb_tally_args;
int tb_tally(tb_ctx *ctx, const tb_tally_args *args, void *stream);

/* The surrogate recurrence over n_batches stored tables (consecutive, each
 * (n_energy + n_angle + 2, m)).  The charge-update fields of the step descriptor
 * are used (m, d_sflag, d_leak_M, d_leak_h, d_g_s, c_slot, floating, driven,
 * q_macro, dx, C_cond, Te) together with its scratch d_rho_prev (m) and d_work (2m). */
typedef struct {
    int n_batches, n_energy, n_angle;
    const int32_t *d_tables;
    const double *d_rE, *d_rA;       /* (n_energy), (n_angle) reweighting factors; NULL = 1 */
    const double *d_leak_MT;         /* (m, m) transpose of the leakage operator (reverse sweep) */
    double *d_rho;                   /* (m) state: in before the first batch, out after the last */
    double *d_scal;                  /* (n_batches, 4) per batch: ion and electron deposit on the
                                        floating conductor, drift (written forward, read reverse) */
    double *d_bottom;                /* (n_batches) reweighted ion deposit on the bottom slots */
    /* Field feedback (reverse sweep only; n_basis = 0 leaves it out): the deposits'
       linear response to the charge state, measured in a basis of n_basis surface-charge
       modes.  d_basis (m, n_basis) orthonormal columns; d_resp_i, d_resp_e (n_sets, m,
       n_basis): ion / electron deposit per unit charge along each mode; d_resp_index
       (n_batches): the response set of each batch, or -1. */
    int n_basis;
    const double *d_basis, *d_resp_i, *d_resp_e;
    const int32_t *d_resp_index;
} tb_adjoint_args;
/* Forward: rho <- recurrence(rho) over the batches; writes d_scal and d_bottom. */
int tb_adjoint_forward(tb_ctx *ctx, const tb_step_desc *step, const tb_adjoint_args *args, void *stream);
/* Reverse over the same batches (their d_scal from the forward):
 *   d_lambda (m): in dJ/d rho after the last batch, out dJ/d rho before the first;
 *   d_gbottom (n_batches): dJ/d bottom deposit of each batch (NULL = 0);
 *   d_grad (n_energy + n_angle): accumulates dJ/d rE, dJ/d rA.
 * Needs the descriptor's d_work (2m) and 2m + 4 + n_basis doubles in d_scratch. */
int tb_adjoint_reverse(tb_ctx *ctx, const tb_step_desc *step, const tb_adjoint_args *args, double *d_lambda,
                       const double *d_gbottom, double *d_grad, double *d_scratch, void *stream);

/* Measured shared-memory load bandwidth of the context's GPU (GB/s, all SMs, 8-byte
 * loads like the FP32 tracer's gathers).  A benchmark helper; synchronises the device. */
int tb_bench_smem(tb_ctx *ctx, double *gbs);
/* Measured random gather bandwidth of whole 32-byte sectors (GB/s, all SMs, read-only
 * path) from a buffer of `bytes` (4 KiB .. 1 GiB, rounded down to a power of two) that
 * stays in L2, like the FP32 tracer's field on grids too large for shared memory.  Allocates and frees
 * its buffer; synchronises the device. */
int tb_bench_l2_gather(tb_ctx *ctx, long long bytes, double *gbs);
/* Self-check of the FP64 tracer's quotients by a divisor with a known reciprocal (cell
 * size, RF period): on n seeded pairs of each of three input families, counts the
 * quotients that differ in any bit from the IEEE division.  Synchronises the device. */
int tb_check_div_by(tb_ctx *ctx, long long n, unsigned long long seed, unsigned long long *mismatches);

#ifdef __cplusplus
}
#endif

#endif /* TRENCH_B200_H */
