// C ABI entry points: contexts, error reporting and argument checks.
// The ABI is declared in include/trench_b200.h.
#include <stdarg.h>
#include <stdlib.h>

#include "tb_internal.cuh"

static char g_create_err[512] = "";

int tb_fail(tb_ctx *ctx, int code, const char *fmt, ...) {
    char *buf = ctx ? ctx->err : g_create_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    return code;
}

int tb_cuda_check(tb_ctx *ctx, cudaError_t e, const char *what) {
    return tb_fail(ctx, TB_ERR_CUDA, "CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
}

extern "C" int tb_version(void) { return 1; }

extern "C" const char *tb_last_error(const tb_ctx *ctx) { return ctx ? ctx->err : g_create_err; }

static int release(tb_ctx *c) {
    if (!c) return TB_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    cudaFree(c->d_vac);
    cudaFree(c->d_field);
    cudaFree(c->d_barrier);
    cudaFree(c->d_rf_field);
    cudaFree(c->d_rf_wave);
    cudaFree(c->d_rf_barrier);
    cudaFree(c->d_queue);
    cudaFree(c->d_claim_rec);
    cudaFree(c->d_claim_key);
    cudaFree(c->d_claim_cls);
    cudaFree(c->d_claim_blk);
    cudaFree(c->d_ion_acc);
    cudaFree(c->d_ion_class);
    cudaFree(c->d_err);
    tb_poisson_free(c->poisson);
    if (prev >= 0) cudaSetDevice(prev);
    delete c;
    return TB_OK;
}

extern "C" int tb_create(tb_ctx **out, int device, int nx, int ny, double dx, const uint8_t *h_vac) {
    if (!out) return tb_fail(nullptr, TB_ERR_ARG, "tb_create: null output pointer");
    *out = nullptr;
    if (nx < 1 || ny < 1 || (long long)nx * ny > (1LL << 30) || !(dx > 0) || !h_vac)
        return tb_fail(nullptr, TB_ERR_ARG, "tb_create: invalid grid (nx=%d, ny=%d, dx=%g)", nx, ny, dx);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) count = 0;
    if (device < 0 || device >= count)
        return tb_fail(nullptr, TB_ERR_DEVICE, "CUDA device %d is not available (%d visible)", device, count);
    tb_ctx *c = new tb_ctx();
    c->device = device;
    c->nx = nx;
    c->ny = ny;
    c->dx = dx;
    cudaError_t e = cudaSetDevice(device);
    cudaDeviceProp prop;
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        tb_cuda_check(nullptr, e, "tb_create");
        release(c);
        return TB_ERR_CUDA;
    }
    snprintf(c->name, sizeof(c->name), "%.120s", prop.name);
    c->num_sms = prop.multiProcessorCount;
    c->max_smem = (int)prop.sharedMemPerBlockOptin;
    c->smem_per_sm = (int)prop.sharedMemPerMultiprocessor;
    const size_t cells = (size_t)nx * ny;
    const size_t padded = (cells + 1) & ~(size_t)1;
    e = cudaMalloc(&c->d_vac, cells);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_field, (size_t)tb_halo_count(nx, ny) * sizeof(tb_fcell));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_barrier, padded * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_queue, 8 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(c->d_vac, h_vac, cells, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->d_barrier, 0, padded * sizeof(float4));
    if (e != cudaSuccess) {
        tb_cuda_check(nullptr, e, "tb_create allocation");
        release(c);
        return TB_ERR_CUDA;
    }
    if (tb_configure_trace_f32(c) != TB_OK) {
        tb_fail(nullptr, TB_ERR_CUDA, "%s", c->err);
        release(c);
        return TB_ERR_CUDA;
    }
    *out = c;
    return TB_OK;
}

extern "C" int tb_destroy(tb_ctx *ctx) { return release(ctx); }

extern "C" int tb_device_info(const tb_ctx *ctx, char *name, int name_len, int *num_sms) {
    if (!ctx) return TB_ERR_ARG;
    if (name && name_len > 0) snprintf(name, name_len, "%s", ctx->name);
    if (num_sms) *num_sms = ctx->num_sms;
    return TB_OK;
}

extern "C" int tb_set_fields(tb_ctx *ctx, const double *d_ex, const double *d_ey, const double *d_phi,
                             const double *d_wface, double vscale, void *stream) {
    if (!ctx) return TB_ERR_ARG;
    if (!d_ex || !d_ey) return tb_fail(ctx, TB_ERR_ARG, "tb_set_fields: Ex and Ey are required");
    if ((d_phi == nullptr) != (d_wface == nullptr))
        return tb_fail(ctx, TB_ERR_ARG, "tb_set_fields: phi and wface must be given together");
    if (!(vscale > 0)) return tb_fail(ctx, TB_ERR_ARG, "tb_set_fields: vscale must be positive");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    return tb_launch_pack_fields(ctx, d_ex, d_ey, d_phi, d_wface, vscale, (cudaStream_t)stream);
}

extern "C" int tb_set_rf_fields(tb_ctx *ctx, const double *d_rf_ex, const double *d_rf_ey, const double *d_rf_phi,
                                const double *d_wface, const double *d_wave, int n_phase, void *stream) {
    if (!ctx) return TB_ERR_ARG;
    if (!d_rf_ex || !d_rf_ey || !d_rf_phi || !d_wave || n_phase < 2)
        return tb_fail(ctx, TB_ERR_ARG, "tb_set_rf_fields: the basis fields, potentials and waveform are required");
    if (!ctx->fields_ready) return tb_fail(ctx, TB_ERR_ARG, "tb_set_rf_fields: call tb_set_fields first");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t cells = (size_t)ctx->nx * ctx->ny;
    if (!ctx->d_rf_field) {
        // allocated on first use: cases without RF never hold these
        TB_CUDA(ctx, cudaMalloc(&ctx->d_rf_field, (size_t)tb_halo_count(ctx->nx, ctx->ny) * sizeof(float4)));
        TB_CUDA(ctx, cudaMalloc(&ctx->d_rf_barrier, 2 * cells * sizeof(float4)));
    }
    if (n_phase > ctx->rf_wave_cap) {
        TB_CUDA(ctx, cudaFree(ctx->d_rf_wave));
        ctx->d_rf_wave = nullptr;
        ctx->rf_wave_cap = 0;
        TB_CUDA(ctx, cudaMalloc(&ctx->d_rf_wave, (size_t)n_phase * sizeof(float4)));
        ctx->rf_wave_cap = n_phase;
    }
    return tb_launch_pack_rf_fields(ctx, d_rf_ex, d_rf_ey, d_rf_phi, d_wface, d_wave, n_phase, (cudaStream_t)stream);
}

// Reads and clears the device error flag (a synchronising copy).
static int check_device_flag(tb_ctx *ctx, cudaStream_t s) {
    int flag = 0;
    TB_CUDA(ctx, cudaMemcpyAsync(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    if (flag != TB_DERR_NONE) {
        TB_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
        return tb_fail(ctx, TB_ERR_KERNEL, "kernel check failed (code %d: %s); the batch's results are partial, "
                       "trace it again", flag,
                       flag == TB_DERR_BULK_TIMEOUT   ? "bulk copy wait gave up"
                       : flag == TB_DERR_BAD_CELL   ? "deposit cell out of range"
                                                    : "absorbed particle outside the surface cells");
    }
    return TB_OK;
}

extern "C" int tb_check(tb_ctx *ctx, void *stream) {
    if (!ctx) return TB_ERR_ARG;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    return check_device_flag(ctx, (cudaStream_t)stream);
}

extern "C" int tb_trace(tb_ctx *ctx, const tb_trace_args *a, int precision, void *stream) {
    if (!ctx) return TB_ERR_ARG;
    if (!a) return tb_fail(ctx, TB_ERR_ARG, "tb_trace: null arguments");
    if (a->n < 0) return tb_fail(ctx, TB_ERR_ARG, "tb_trace: negative particle count");
    if (!(a->cfl > 0 && a->cfl <= 1) || a->max_steps < 1)
        return tb_fail(ctx, TB_ERR_ARG, "CUDA tracing needs 0 < cfl <= 1 and max_steps >= 1");
    if (a->step_budget < 1) return tb_fail(ctx, TB_ERR_ARG, "tb_trace: step_budget must be >= 1");
    if (a->n == 0) return TB_OK;
    if (!a->d_x || !a->d_y || !a->d_vx || !a->d_vy || !a->d_qm || !a->d_spc || !a->d_counts || !a->d_totals ||
        !a->d_status || !a->d_steps)
        return tb_fail(ctx, TB_ERR_ARG, "tb_trace: a required array is missing");
    if ((a->d_phi == nullptr) != (a->d_wface == nullptr))
        return tb_fail(ctx, TB_ERR_ARG, "tb_trace: phi and wface must be given together");
    if (a->n_phase < 0 || (a->n_phase > 0 && (a->n_phase < 2 || !a->d_rf_ex || !a->d_rf_ey || !a->d_rf_phi ||
                                                !a->d_wave || !a->d_clock || !(a->period > 0) ||
                                                !(a->dt_max > 0))))
        return tb_fail(ctx, TB_ERR_ARG, "tb_trace: invalid RF clock arguments");
    if (a->record && (!a->d_endpoints || a->path_stride < 1))
        return tb_fail(ctx, TB_ERR_ARG, "tb_trace: record needs endpoints and a path stride");
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == TB_PRECISION_F64) {
        if (!a->d_ex || !a->d_ey) return tb_fail(ctx, TB_ERR_ARG, "tb_trace: FP64 tracing needs Ex and Ey");
        return tb_launch_trace_f64(ctx, a, s);
    }
    if (precision == TB_PRECISION_F32) {
        if (a->record) return tb_fail(ctx, TB_ERR_ARG, "tb_trace: record needs precision F64");
        if (!ctx->fields_ready) return tb_fail(ctx, TB_ERR_ARG, "tb_trace: call tb_set_fields first");
        if (a->n_phase > 0 && (!ctx->rf_ready || ctx->rf_vscale != ctx->vscale))
            return tb_fail(ctx, TB_ERR_ARG, "tb_trace: FP32 with the RF clock needs tb_set_rf_fields after tb_set_fields");
        if (a->n_phase > 0 && (a->d_wave != ctx->rf_wave_src || a->n_phase != ctx->rf_n_phase))
            return tb_fail(ctx, TB_ERR_ARG, "tb_trace: the waveform differs from the one given to tb_set_rf_fields");
        return tb_launch_trace_f32(ctx, a, s);
    }
    return tb_fail(ctx, TB_ERR_ARG, "tb_trace: unknown precision %d", precision);
}
