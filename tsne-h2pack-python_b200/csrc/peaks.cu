// Measured compute ceilings of this GPU for the roofline of the non-tensor kernels (no
// counterpart in the reference): FP32 fused multiply-add throughput, scalar (FFMA) and in the
// paired form (fma.rn.f32x2, two lanes of data per instruction) that the 2D near-field kernel
// issues, and the MUFU reciprocal rate the kernel (1 + r^2)^-2 needs once per pair.
#include <cuda_runtime.h>
#include <stdio.h>

#include "common.cuh"
#include "../../include/tsne_h2pack.h"

using namespace tsne;

namespace {

constexpr int PEAK_CHAINS = 8;      // independent accumulators per thread (FMA latency hiding)
constexpr int PEAK_ITERS = 16384;
constexpr int PEAK_THREADS = 256;
constexpr int PEAK_BLOCKS = 148 * 8;

__global__ void __launch_bounds__(PEAK_THREADS) k_peak_ffma(float seed, float *out)
{
    float a[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) a[c] = seed + threadIdx.x * 1e-7f + c;
    const float m = 0.9999f, b = 1e-6f;
    for (int it = 0; it < PEAK_ITERS; it++)
#pragma unroll
        for (int c = 0; c < PEAK_CHAINS; c++) a[c] = fmaf(a[c], m, b);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) s += a[c];
    if (s == 1234.5f) out[blockIdx.x] = s;   // keeps the loop live; never true in practice
}

__global__ void __launch_bounds__(PEAK_THREADS) k_peak_ffma2(float seed, float *out)
{
    F2 a[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) a[c] = f2_pack(seed + threadIdx.x * 1e-7f + c, seed - c);
    const F2 m = f2_pack(0.9999f, 0.9999f), b = f2_pack(1e-6f, 1e-6f);
    for (int it = 0; it < PEAK_ITERS; it++)
#pragma unroll
        for (int c = 0; c < PEAK_CHAINS; c++) a[c] = f2_fma(a[c], m, b);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) {
        float lo, hi;
        f2_unpack(a[c], lo, hi);
        s += lo + hi;
    }
    if (s == 1234.5f) out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(PEAK_THREADS) k_peak_rcp(float seed, float *out)
{
    float a[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) a[c] = 1.5f + seed + threadIdx.x * 1e-7f + c;
    for (int it = 0; it < PEAK_ITERS / 4; it++)
#pragma unroll
        for (int c = 0; c < PEAK_CHAINS; c++) a[c] = fast_rcp(a[c]) + 1.0f;
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) s += a[c];
    if (s == 1234.5f) out[blockIdx.x] = s;
}

template <typename K>
double time_ms(K kernel, float *out, cudaStream_t st)
{
    cudaEvent_t e0, e1;
    TSNE_CUDA_CHECK(cudaEventCreate(&e0));
    TSNE_CUDA_CHECK(cudaEventCreate(&e1));
    kernel<<<PEAK_BLOCKS, PEAK_THREADS, 0, st>>>(0.5f, out);   // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        TSNE_CUDA_CHECK(cudaEventRecord(e0, st));
        kernel<<<PEAK_BLOCKS, PEAK_THREADS, 0, st>>>(0.5f, out);
        TSNE_CUDA_CHECK(cudaEventRecord(e1, st));
        TSNE_CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        TSNE_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace

extern "C" TSNE_API int tsne_measure_compute_peaks(double *ffma_tflops, double *ffma2_tflops, double *rcp_tops)
{
    try {
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        float *out = nullptr;
        TSNE_CUDA_CHECK(cudaMalloc(&out, sizeof(float) * PEAK_BLOCKS));
        const double threads = (double)PEAK_BLOCKS * PEAK_THREADS;
        const double fma_ops = threads * PEAK_ITERS * PEAK_CHAINS;
        const double t1 = time_ms(k_peak_ffma, out, st);
        const double t2 = time_ms(k_peak_ffma2, out, st);
        const double t3 = time_ms(k_peak_rcp, out, st);
        if (ffma_tflops) *ffma_tflops = 2.0 * fma_ops / (t1 * 1e-3) / 1e12;
        if (ffma2_tflops) *ffma2_tflops = 4.0 * fma_ops / (t2 * 1e-3) / 1e12;
        if (rcp_tops) *rcp_tops = (threads * (PEAK_ITERS / 4) * PEAK_CHAINS) / (t3 * 1e-3) / 1e12;
        cudaFree(out);
        cudaStreamDestroy(st);
    } catch (const CudaError &) {
        return -2;
    }
    return 0;
}
