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
    /* circuit_rf in-flight clock (F64 only); n_phase = 0 disables */
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
    int64_t *d_totals;               /* [4] escaped ions, escaped electrons, lost, particle-steps;
                                        accumulated */
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

/* Trace particles until absorbed, escaped or max_steps; deposit hits into
 * d_counts with integer atomics.  Replaces the chunk loop, kernel launch and host
 * bincount of CudaTracer._trace (trench_cuda.py:100-122) and the kernel
 * trace_particles (trench_trace.cu:70-193). */
int tb_trace(tb_ctx *ctx, const tb_trace_args *args, int precision, void *stream);

/* Synchronise `stream`, then read and clear the context's device-side check flag:
 * TB_ERR_KERNEL if a kernel recorded a failed bound (a deposit cell outside the
 * grid, a bulk copy that did not complete in its bounded wait). */
int tb_check(tb_ctx *ctx, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TRENCH_B200_H */
