// Internal declarations shared by the trench_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/trench_b200.h"

// Device-side error codes written to tb_ctx::d_err (first error wins).
#define TB_DERR_NONE 0
#define TB_DERR_BULK_TIMEOUT 1   // bounded wait on a bulk-copy barrier gave up
#define TB_DERR_BAD_CELL 2       // a deposit cell fell outside the grid
#define TB_DERR_OFF_SURFACE 3    // an absorbed particle was counted outside the surface cells

// Packed FP32 field cell: E*vac in cell units; bit 0 of .x carries the vacuum flag.
struct __align__(8) tb_fcell {
    float ex, ey;
};

struct tb_poisson;
void tb_poisson_free(tb_poisson *ps);

struct tb_ctx {
    int device = 0;
    int nx = 0, ny = 0;
    double dx = 0;
    int num_sms = 0;
    char name[128] = {0};
    uint8_t *d_vac = nullptr;            // (nx*ny)
    tb_fcell *d_field = nullptr;         // packed FP32 field, padded to 16 bytes
    float4 *d_barrier = nullptr;         // per solid cell: barrier toward W, E, S, N neighbour
    unsigned long long *d_queue = nullptr;  // scratch: work counters
    int *d_err = nullptr;                // scratch: device error flag
    double vscale = 1e5;                 // velocity unit of the FP32 state, m/s
    int fields_ready = 0;
    int max_smem = 0;                    // opt-in shared memory per block (bytes)
    int smem_attr_bytes = 0;             // dynamic shared memory set on the FP32 tracer
    tb_poisson *poisson = nullptr;        // multigrid hierarchy (tb_poisson_setup)
    char err[512] = {0};
};

// Records a message on the context and returns `code`.
int tb_fail(tb_ctx *ctx, int code, const char *fmt, ...);
// Turns a CUDA error into TB_ERR_CUDA with the call site in the message.
int tb_cuda_check(tb_ctx *ctx, cudaError_t e, const char *what);

#define TB_CUDA(ctx, call)                                          \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return tb_cuda_check(ctx, e_, #call); \
    } while (0)

// Launchers implemented per translation unit.
int tb_launch_trace_f64(tb_ctx *ctx, const tb_trace_args *a, cudaStream_t s);
int tb_launch_trace_f32(tb_ctx *ctx, const tb_trace_args *a, cudaStream_t s);
int tb_configure_trace_f32(tb_ctx *ctx);
int tb_launch_pack_fields(tb_ctx *ctx, const double *ex, const double *ey, const double *phi,
                          const double *wface, double vscale, cudaStream_t s);

// Periodic index helpers.
__host__ __device__ __forceinline__ int tb_wrap(int i, int n) {
    return i < 0 ? i + n : (i >= n ? i - n : i);
}
__host__ __device__ __forceinline__ int tb_clip(int i, int n) {
    return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
}
