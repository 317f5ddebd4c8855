// Bandwidth microbenchmarks for the FP32 tracer's roofline denominators: shared-memory
// loads (its bilinear gathers are 8-byte shared-memory loads) and random 32-byte
// sector gathers from an L2-resident global buffer (the path of grids too large for
// shared memory).
#include "tb_internal.cuh"

namespace {

__global__ void __launch_bounds__(1024, 1) k_smem_read(int words, int iters, float *sink) {
    extern __shared__ float2 buf[];
    for (int i = threadIdx.x; i < words; i += blockDim.x) buf[i] = make_float2((float)i, 1.f);
    __syncthreads();
    float2 acc = make_float2(0.f, 0.f);
    int idx = threadIdx.x;
    const int mask = words - 1;  // words is a power of two
    const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(buf));
#pragma unroll 8
    for (int it = 0; it < iters; ++it) {
        float vx, vy;
        // volatile: every iteration issues its load (no reuse across iterations)
        asm volatile("ld.volatile.shared.v2.f32 {%0, %1}, [%2];" : "=f"(vx), "=f"(vy) : "r"(base + 8u * idx));
        acc.x += vx;
        acc.y += vy;
        idx = (idx + blockDim.x) & mask;
    }
    if (acc.x == -1.f) sink[blockIdx.x] = acc.y;  // keeps the loads live
}

// Random gathers of whole 32-byte sectors (two 16-byte loads each, the unit in which L2
// serves a request) from a global buffer small enough to stay in L2, read-only path as
// the FP32 tracer's global-memory field; four independent chains per thread.
__global__ void __launch_bounds__(1024, 1) k_l2_gather(const float4 *__restrict__ buf, unsigned mask, int iters,
                                                       float *sink) {
    unsigned i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u, i1 = i0 ^ 0x9e3779b9u,
             i2 = i0 ^ 0x7f4a7c15u, i3 = i0 ^ 0x94d049bbu;
    float acc = 0.f;
#pragma unroll 2
    for (int it = 0; it < iters; ++it) {
        const unsigned s0 = 2u * (i0 & mask), s1 = 2u * (i1 & mask), s2 = 2u * (i2 & mask), s3 = 2u * (i3 & mask);
        const float4 a0 = __ldg(buf + s0), a1 = __ldg(buf + s0 + 1), b0 = __ldg(buf + s1), b1 = __ldg(buf + s1 + 1);
        const float4 c0 = __ldg(buf + s2), c1 = __ldg(buf + s2 + 1), d0 = __ldg(buf + s3), d1 = __ldg(buf + s3 + 1);
        acc += ((a0.x + a1.w) + (b0.y + b1.z)) + ((c0.z + c1.y) + (d0.w + d1.x));
        i0 = i0 * 1664525u + 1013904223u;
        i1 = i1 * 1664525u + 1013904223u;
        i2 = i2 * 1664525u + 1013904223u;
        i3 = i3 * 1664525u + 1013904223u;
    }
    if (acc == -1.f) sink[blockIdx.x] = acc;  // keeps the loads live
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// tb_div_by(a, b, RN(1/b)) against a / b on n seeded pairs of one family: 0 any
// significands with exponents within +-60, 1 positions 0-10 um over cell sizes
// 0.1-10 nm, 2 divisors with significands near all-ones or near one.
__global__ void k_check_div_by(long long n, unsigned long long seed, int family, unsigned long long *bad) {
    unsigned long long mine = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint64_t h1 = mix64(2 * (uint64_t)i + seed * 0x9E3779B97F4A7C15ULL);
        const uint64_t h2 = mix64(2 * (uint64_t)i + 1 + seed * 0x9E3779B97F4A7C15ULL);
        double a, b;
        if (family == 0) {
            a = __longlong_as_double((long long)((h1 & 0x000fffffffffffffULL) | ((uint64_t)(1023 - 60 + (h1 >> 52) % 121) << 52)));
            b = __longlong_as_double((long long)((h2 & 0x000fffffffffffffULL) | ((uint64_t)(1023 - 60 + (h2 >> 52) % 121) << 52)));
            if (h1 >> 63) a = -a;
        } else if (family == 1) {
            b = 1e-10 * (1.0 + 99.0 * (double)(h2 >> 11) * 0x1p-53);
            a = 1e-5 * ((double)(h1 >> 11) * 0x1p-53 - 0.01);
        } else {
            const uint64_t m = (h2 & 1) ? (0x000fffffffffffffULL - (h2 >> 40)) : (h2 >> 40);
            b = __longlong_as_double((long long)(m | (1023ULL << 52)));
            a = __longlong_as_double((long long)((h1 & 0x000fffffffffffffULL) | ((uint64_t)(1023 - 5 + (h1 >> 52) % 11) << 52)));
        }
        const double q0 = a / b, q1 = tb_div_by(a, b, 1.0 / b);
        mine += __double_as_longlong(q0) != __double_as_longlong(q1);
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(bad, mine);
}

}  // namespace

extern "C" int tb_check_div_by(tb_ctx *ctx, long long n, unsigned long long seed, unsigned long long *mismatches) {
    if (!ctx || !mismatches || n < 0) return TB_ERR_ARG;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned long long *bad = nullptr;
    TB_CUDA(ctx, cudaMalloc(&bad, sizeof(unsigned long long)));
    TB_CUDA(ctx, cudaMemset(bad, 0, sizeof(unsigned long long)));
    for (int family = 0; family < 3; ++family)
        k_check_div_by<<<ctx->num_sms * 8, 256>>>(n, seed + (unsigned long long)family, family, bad);
    const cudaError_t e = cudaGetLastError();
    unsigned long long h = 0;
    const cudaError_t c = cudaMemcpy(&h, bad, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(bad);
    TB_CUDA(ctx, e);
    TB_CUDA(ctx, c);
    *mismatches = h;
    return TB_OK;
}

extern "C" int tb_bench_l2_gather(tb_ctx *ctx, long long bytes, double *gbs) {
    if (!ctx || !gbs || bytes < 4096 || bytes > (1LL << 30)) return TB_ERR_ARG;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned long long sectors = 1;
    while (sectors * 2 * 32 <= (unsigned long long)bytes) sectors *= 2;  // largest power of two that fits
    const int threads = 1024, iters = 1 << 11;
    const int blocks = ctx->num_sms;
    float4 *buf = nullptr;
    float *sink = nullptr;
    cudaEvent_t a, b;
    TB_CUDA(ctx, cudaMalloc(&buf, sectors * 32));
    TB_CUDA(ctx, cudaMemset(buf, 0, sectors * 32));
    TB_CUDA(ctx, cudaMalloc(&sink, blocks * sizeof(float)));
    TB_CUDA(ctx, cudaEventCreate(&a));
    TB_CUDA(ctx, cudaEventCreate(&b));
    k_l2_gather<<<blocks, threads>>>(buf, (unsigned)(sectors - 1), iters, sink);  // warm-up: the buffer enters L2
    TB_CUDA(ctx, cudaGetLastError());
    TB_CUDA(ctx, cudaDeviceSynchronize());
    TB_CUDA(ctx, cudaEventRecord(a));
    k_l2_gather<<<blocks, threads>>>(buf, (unsigned)(sectors - 1), iters, sink);
    TB_CUDA(ctx, cudaGetLastError());
    TB_CUDA(ctx, cudaEventRecord(b));
    TB_CUDA(ctx, cudaEventSynchronize(b));
    float ms = 0;
    TB_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    cudaFree(buf);
    *gbs = (double)blocks * threads * (double)iters * 4 * 32 / (ms * 1e-3) / 1e9;
    return TB_OK;
}

extern "C" int tb_bench_smem(tb_ctx *ctx, double *gbs) {
    if (!ctx || !gbs) return TB_ERR_ARG;
    TB_CUDA(ctx, cudaSetDevice(ctx->device));
    const int words = 4096;  // 32 KiB of float2 (below the default dynamic limit)
    const int threads = 1024, iters = 1 << 14;
    const int blocks = ctx->num_sms;
    float *sink = nullptr;
    cudaEvent_t a, b;
    TB_CUDA(ctx, cudaMalloc(&sink, blocks * sizeof(float)));
    TB_CUDA(ctx, cudaEventCreate(&a));
    TB_CUDA(ctx, cudaEventCreate(&b));
    k_smem_read<<<blocks, threads, words * sizeof(float2)>>>(words, iters, sink);  // warm-up
    TB_CUDA(ctx, cudaGetLastError());
    TB_CUDA(ctx, cudaDeviceSynchronize());
    TB_CUDA(ctx, cudaEventRecord(a));
    k_smem_read<<<blocks, threads, words * sizeof(float2)>>>(words, iters, sink);
    TB_CUDA(ctx, cudaGetLastError());
    TB_CUDA(ctx, cudaEventRecord(b));
    TB_CUDA(ctx, cudaEventSynchronize(b));
    float ms = 0;
    TB_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    *gbs = (double)blocks * threads * (double)iters * sizeof(float2) / (ms * 1e-3) / 1e9;
    return TB_OK;
}
