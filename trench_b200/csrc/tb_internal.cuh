// Internal declarations shared by the trench_b200 CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/trench_b200.h"

// Device-side error codes written to tb_ctx::d_err (first error wins).
#define TB_DERR_NONE 0
#define TB_DERR_BULK_TIMEOUT 1   // bounded wait on a bulk-copy barrier gave up: the CTA returned
                                 // untraced, so the batch's outputs are partial
#define TB_DERR_BAD_CELL 2       // a deposit cell fell outside the grid
#define TB_DERR_OFF_SURFACE 3    // an absorbed particle was counted outside the surface cells

// Packed FP32 field cell: E*vac in cell units; bit 0 of .x carries the vacuum flag.
struct __align__(8) tb_fcell {
    float ex, ey;
};

// Packed FP32 field with a one-cell halo: padded cell (i, j), i in [-1, nx],
// j in [-1, ny], lives at (i + 1) * (ny + 2) + (j + 1).  Column -1 repeats
// column nx-1 and column nx repeats column 0 (x periodic); row -1 repeats row 0
// and row ny repeats row ny-1 (the reference clips y indices,
// trench_charging_2d.py:502-505).  Bilinear corners then need no wrap or clip.
__host__ __device__ __forceinline__ int tb_halo_count(int nx, int ny) {
    const int n = (nx + 2) * (ny + 2);
    return (n + 1) & ~1;  // even count: whole 16-byte units for the bulk copy
}

// Physical column / row of padded column pi / row pj (x periodic, rows clipped).
__host__ __device__ __forceinline__ int tb_pad_col(int pi, int nx) {
    return pi == 0 ? nx - 1 : (pi == nx + 1 ? 0 : pi - 1);
}
__host__ __device__ __forceinline__ int tb_pad_row(int pj, int ny) {
    return pj == 0 ? 0 : (pj == ny + 1 ? ny - 1 : pj - 1);
}

// True if the bilinear quad whose lower-left corner is padded cell (pi, pj) -- the
// corners (pi, pj), (pi+1, pj), (pi, pj+1), (pi+1, pj+1) -- has four vacuum cells.
// A step of less than half a cell that starts inside such a quad ends in one of its
// corner cells, so it cannot reach a wall, and its vacuum weights sum to one.
// Quads beyond the last corner column or row (never a particle's quad) report false.
__device__ __forceinline__ bool tb_quad_vacuum(const uint8_t *vac, int nx, int ny, int pi, int pj) {
    if (pi > nx || pj > ny) return false;
    const int c0 = tb_pad_col(pi, nx) * ny, c1 = tb_pad_col(pi + 1, nx) * ny;
    const int r0 = tb_pad_row(pj, ny), r1 = tb_pad_row(pj + 1, ny);
    return vac[c0 + r0] && vac[c0 + r1] && vac[c1 + r0] && vac[c1 + r1];
}

// Packed tracer cell: E*vac scaled to cell units, bit 0 of ex = vacuum (one-ulp
// perturbation of the FP32 value; a flagged zero becomes the smallest denormal, which
// flushes to zero in the tracer's arithmetic).  Bit 0 of ey is set per padded position
// by tb_store_packed (the quad flag).
__device__ __forceinline__ tb_fcell tb_pack_cell(double ex, double ey, bool vacuum, double scale) {
    const double v = vacuum ? 1.0 : 0.0;
    uint32_t bx = __float_as_uint((float)(ex * v * scale));
    bx = vacuum ? (bx | 1u) : (bx & ~1u);
    return tb_fcell{__uint_as_float(bx), (float)(ey * v * scale)};
}

// Writes the packed value of cell (ix, iy) and its halo copies.
template <typename T>
__device__ __forceinline__ void tb_store_halo(T *out, int nx, int ny, int ix, int iy, T v) {
    const int P = ny + 2;
    int cs[3], rs[3], nc = 0, nr = 0;
    cs[nc++] = ix + 1;
    if (ix == nx - 1) cs[nc++] = 0;
    if (ix == 0) cs[nc++] = nx + 1;
    rs[nr++] = iy + 1;
    if (iy == 0) rs[nr++] = 0;
    if (iy == ny - 1) rs[nr++] = ny + 1;
    for (int a = 0; a < nc; ++a)
        for (int b = 0; b < nr; ++b) out[cs[a] * P + rs[b]] = v;
}

// tb_store_halo for the packed tracer field: every padded copy of cell (ix, iy) gets the
// quad flag of its own padded position in bit 0 of ey.
__device__ __forceinline__ void tb_store_packed(tb_fcell *out, const uint8_t *vac, int nx, int ny, int ix, int iy,
                                                tb_fcell v) {
    const int P = ny + 2;
    int cs[3], rs[3], nc = 0, nr = 0;
    cs[nc++] = ix + 1;
    if (ix == nx - 1) cs[nc++] = 0;
    if (ix == 0) cs[nc++] = nx + 1;
    rs[nr++] = iy + 1;
    if (iy == 0) rs[nr++] = 0;
    if (iy == ny - 1) rs[nr++] = ny + 1;
    const uint32_t by = __float_as_uint(v.ey) & ~1u;
    for (int a = 0; a < nc; ++a)
        for (int b = 0; b < nr; ++b) {
            const uint32_t q = tb_quad_vacuum(vac, nx, ny, cs[a], rs[b]) ? 1u : 0u;
            out[cs[a] * P + rs[b]] = tb_fcell{v.ex, __uint_as_float(by | q)};
        }
}

struct tb_poisson;
void tb_poisson_free(tb_poisson *ps);

// Learned claim order of the FP32 tracer (tb_set_claim_order 2): ions are binned by
// starting column band and direction, each bin's mean step count is learned from the
// previous trace, and the particles are claimed electrons first, then ions longest
// predicted first, through a table of claim records written in that order.
constexpr int TB_ORDER_ION_BINS = 512;   // 128 column bands x 4 direction bands
constexpr int TB_ORDER_CLASSES = 16;     // class 0 electrons, 1..15 ions by predicted length

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
    int smem_per_sm = 0;                 // shared memory of one SM (bytes)
    int tune_threads = 0;                // FP32 tracer CTA size (tb_set_tuning), 0 = by batch size
    int tune_ctas_per_sm = 1;            // FP32 tracer CTAs per SM
    int tune_reverse = 0;                // FP32 tracer claim order: 0 index, 1 from the last index down, 2 learned
    uint4 *d_claim_rec = nullptr;        // learned order: claim records (2 x uint4 per eligible particle)
    uint16_t *d_claim_key = nullptr;     // learned order: each particle's ion bin (0xffff: electron / not traced)
    long long claim_cap = 0;             // particles the two arrays above hold
    unsigned *d_claim_cls = nullptr;     // learned order: number of claim records
    unsigned *d_claim_blk = nullptr;     // learned order: per block and class, particle count then start
    unsigned *d_ion_acc = nullptr;       // learned order: per ion bin step sum and count of the last trace
    uint8_t *d_ion_class = nullptr;      // learned order: class of each ion bin for the next trace
    float4 *d_rf_field = nullptr;        // circuit_rf basis fields (exs, eys, exm, eym) x vac, halo-padded
    float4 *d_rf_barrier = nullptr;      // (2, nx*ny) per-face wall barrier of each basis potential
    int rf_ready = 0;
    double rf_vscale = 0;                // velocity unit the basis fields were packed with
    float4 *d_rf_wave = nullptr;         // waveform per table interval: (vs_i, vm_i, vs_i+1 - vs_i, vm_i+1 - vm_i)
    int rf_wave_cap = 0;                 // intervals allocated
    int rf_n_phase = 0;                  // intervals packed
    const double *rf_wave_src = nullptr; // the FP64 waveform they were packed from
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
int tb_launch_pack_rf_fields(tb_ctx *ctx, const double *rf_ex, const double *rf_ey, const double *rf_phi,
                             const double *wface, const double *wave, int n_phase, cudaStream_t s);

// One case's per-batch update as the case-pack update kernels read it (device array,
// one entry per case): its step descriptor, grid and packed tracer-field outputs.
struct tb_pack_step_entry {
    tb_step_desc d;
    int nx, ny;
    const uint8_t *vac;
    double scale_e, scale_phi;
    tb_fcell *field;
    float4 *bar;
    int *err;
};

// Per-batch update of every case of a pack (tb_step.cu): set once from one descriptor
// per case, then run as one launch per stage.
struct tb_pack_steps;
int tb_pack_steps_set(tb_pack_steps **ps, int n, tb_ctx *const *ctxs, const tb_step_desc *descs, char *err,
                      size_t errlen);
int tb_pack_steps_run(tb_pack_steps *ps, cudaStream_t s, char *err, size_t errlen);
void tb_pack_steps_free(tb_pack_steps *ps);

// Deposits one particle into counts[key] (key = species * cells + cell).  Warp-aggregated:
// the lanes of the warp that deposit into the same key at this point add once, with
// the number of such lanes.  The counts are integers, so the result is exact and
// independent of the order of the additions.
__device__ __forceinline__ void tb_deposit(int32_t *counts, size_t key) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, (unsigned long long)key);
    if ((int)(threadIdx.x & 31u) == __ffs(peers) - 1) atomicAdd(counts + key, __popc(peers));
}

// a / b rounded to nearest for a divisor b whose rounded reciprocal rb = RN(1/b) is known:
// q = RN(a rb) is within one ulp of a/b, and one correction with the exact remainder
// a - b q (a fused multiply-add) gives the correctly rounded quotient (Markstein's
// theorem: P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990).  Three dependent operations in place of a full
// division; valid while no intermediate overflows or underflows.  tb_check_div_by compares
// it with the division on the device.
__device__ __forceinline__ double tb_div_by(double a, double b, double rb) {
    const double q = __dmul_rn(a, rb);
    const double r = fma(-q, b, a);
    return fma(r, rb, q);
}

// Periodic index helpers.
__host__ __device__ __forceinline__ int tb_wrap(int i, int n) {
    return i < 0 ? i + n : (i >= n ? i - n : i);
}
__host__ __device__ __forceinline__ int tb_clip(int i, int n) {
    return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
}
