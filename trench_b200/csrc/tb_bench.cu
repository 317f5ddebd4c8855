// Shared-memory load bandwidth microbenchmark: the roofline denominator of the
// FP32 tracer, whose bilinear gathers are 8-byte shared-memory loads.
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

}  // namespace

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
