// tsne_exact_repulsion_static: the exact O(N^2) repulsive force for callers that cannot
// allocate device memory.
//
// Some callers must not allocate: code that runs under a caller-owned memory budget (a
// serving process that has carved HBM up front and may not grow), code that runs inside a
// region where an allocation's implicit device synchronisation is not acceptable, or hosts
// whose allocator is not the CUDA runtime's. This entry point takes device pointers for its
// input and outputs and keeps its scratch (per-point force sums and the per-block partial
// sums of Z) in a file-scope __device__ array of fixed size, so it calls no cudaMalloc,
// cudaFree or any other allocating routine.
//
// Numerics. The force and Z are those of the reference's exact branch
// (src/tsne_h2pack.c:404-491): K_ij = (1 + |y_i - y_j|^2)^-2, F_i = (4 / Z) sum_{j != i}
// K_ij (y_i - y_j) and Z = sum_{i != j} (1 + |y_i - y_j|^2)^-1. The reference reaches Z
// through the identity Z = sum s + 2 sum |y|^2 s - 2 sum y.v and the force through
// y_i s_i - v_i; both subtract large, nearly equal terms when the embedding is wide, which
// FP64 absorbs and FP32 does not. Here each pair contributes its own difference vector and its
// own (1 + r^2)^-1, so nothing cancels: pair terms are FP32, a thread's sums over a tile of
// 256 sources are FP32, the sums over tiles FP64, and Z is a fixed-order FP64 sum of
// per-block partials (the result is the same bits on every call).
//
// The scratch array exists once per device and is shared by every call on that device: calls
// that overlap on the GPU (two streams at once, or two host threads) race on it. Every
// element a call reads is written earlier by the same call, so no clearing is needed.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "common.cuh"
#include "../../include/tsne_h2pack.h"

namespace {

using namespace tsne;

constexpr int NA_MAX_POINTS = 65536;                       // largest n_point accepted
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_BLOCKS = NA_MAX_POINTS / NA_THREADS;  // Z partials, one per block of targets
// g: NA_MAX_POINTS float4 (force sums, w unused), then NA_MAX_BLOCKS doubles of Z partials
constexpr size_t NA_SCRATCH_FLOATS = (size_t)NA_MAX_POINTS * 4 + (size_t)NA_MAX_BLOCKS * 2;

static __device__ __align__(256) float na_scratch[NA_SCRATCH_FLOATS];

constexpr int NA_MAX_DEVICES = 64;
float *na_ptr[NA_MAX_DEVICES] = {nullptr};
std::mutex na_mu;

template <int D>
__device__ __forceinline__ void load_pt(const float *Y, int i, float (&p)[D])
{
#pragma unroll
    for (int k = 0; k < D; k++) p[k] = Y[(size_t)i * D + k];
}

// Per target i (a thread each): g_i = sum_{j != i} K_ij (y_i - y_j), and the block's sum of
// q_i = sum_{j != i} (1 + r_ij^2)^-1; sources staged 256 at a time in shared memory.
template <int D>
__global__ void __launch_bounds__(NA_THREADS) k_na_pairs(int n, const float *__restrict__ Y,
                                                         float4 *__restrict__ g, double *__restrict__ zpart)
{
    __shared__ float sh[NA_THREADS][D];
    __shared__ double red[NA_THREADS];
    const int i = blockIdx.x * NA_THREADS + threadIdx.x;
    float yi[D];
    for (int k = 0; k < D; k++) yi[k] = 0.f;
    if (i < n) load_pt<D>(Y, i, yi);
    double Q = 0.0, G[D];
    for (int k = 0; k < D; k++) G[k] = 0.0;
    for (int base = 0; base < n; base += NA_THREADS) {
        __syncthreads();
        if (base + (int)threadIdx.x < n)
            for (int k = 0; k < D; k++) sh[threadIdx.x][k] = Y[(size_t)(base + threadIdx.x) * D + k];
        __syncthreads();
        const int cnt = min(NA_THREADS, n - base);
        float tq = 0.f, tg[D];
        for (int k = 0; k < D; k++) tg[k] = 0.f;
        for (int j = 0; j < cnt; j++) {
            float df[D], r2 = 0.f;
#pragma unroll
            for (int k = 0; k < D; k++) { df[k] = yi[k] - sh[j][k]; r2 = fmaf(df[k], df[k], r2); }
            float w = 1.0f / (1.0f + r2);
            w = (base + j == i) ? 0.f : w;
            tq += w;
            const float kk = w * w;
#pragma unroll
            for (int k = 0; k < D; k++) tg[k] = fmaf(kk, df[k], tg[k]);
        }
        Q += tq;
        for (int k = 0; k < D; k++) G[k] += tg[k];
    }
    if (i < n) {
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        o.x = (float)G[0];
        o.y = (float)G[1];
        if (D == 3) o.z = (float)G[D - 1];
        g[i] = o;
    }
    red[threadIdx.x] = (i < n) ? Q : 0.0;
    __syncthreads();
    for (int st = NA_THREADS / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) zpart[blockIdx.x] = red[0];
}

// Z = fixed-order sum of the block partials (every block sums them the same way), then
// F_i = (4 / Z) g_i. A Z that is not positive and finite (the embedding holds a NaN or an
// infinity) is stored as it is and F is set to zero.
template <int D>
__global__ void __launch_bounds__(NA_THREADS) k_na_force(int n, int nblk, const float4 *__restrict__ g,
                                                         const double *__restrict__ zpart, float *__restrict__ F,
                                                         double *__restrict__ Zout)
{
    __shared__ double red[NA_THREADS];
    red[threadIdx.x] = (int)threadIdx.x < nblk ? zpart[threadIdx.x] : 0.0;
    __syncthreads();
    for (int st = NA_THREADS / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    const double Z = red[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) *Zout = Z;
    const bool ok = Z > 0.0 && isfinite(Z);
    const double c = ok ? 4.0 / Z : 0.0;
    const int i = blockIdx.x * NA_THREADS + threadIdx.x;
    if (i < n) {
        const float4 gi = ok ? g[i] : make_float4(0.f, 0.f, 0.f, 0.f);   // 0 * NaN would be NaN
        F[(size_t)i * D + 0] = (float)(c * gi.x);
        F[(size_t)i * D + 1] = (float)(c * gi.y);
        if (D == 3) F[(size_t)i * D + D - 1] = (float)(c * gi.z);
    }
}

// Device address of the scratch array on the current device, looked up once per device with
// that device current (the host-side name of a __device__ array is not a device address).
float *scratch_address(int *err)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) { *err = -2; return nullptr; }
    std::lock_guard<std::mutex> lock(na_mu);
    if (na_ptr[dev] == nullptr) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, na_scratch);
        if (e != cudaSuccess || p == nullptr) {
            fprintf(stderr, "tsne_exact_repulsion_static: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            *err = -2;
            return nullptr;
        }
        na_ptr[dev] = static_cast<float *>(p);
    }
    return na_ptr[dev];
}

}  // namespace

extern "C" TSNE_API int tsne_exact_repulsion_static(const float *Y, int n_point, int low_dim, float *F, double *Z,
                                                    void *stream)
{
    if (Y == nullptr || F == nullptr || Z == nullptr || (low_dim != 2 && low_dim != 3)) {
        fprintf(stderr, "tsne_exact_repulsion_static: bad arguments\n");
        return -1;
    }
    if (n_point < 2 || n_point > NA_MAX_POINTS) {
        fprintf(stderr, "tsne_exact_repulsion_static: n_point = %d is outside [2, %d] (the size of its fixed "
                        "scratch array)\n", n_point, NA_MAX_POINTS);
        return -1;
    }
    const uintptr_t y0 = (uintptr_t)Y, f0 = (uintptr_t)F, bytes = (uintptr_t)n_point * low_dim * sizeof(float);
    if (y0 < f0 + bytes && f0 < y0 + bytes) {
        fprintf(stderr, "tsne_exact_repulsion_static: F overlaps Y (the force cannot be written in place)\n");
        return -1;
    }
    int err = 0;
    float *scratch = scratch_address(&err);
    if (scratch == nullptr) return err;
    float4 *g = reinterpret_cast<float4 *>(scratch);
    double *zpart = reinterpret_cast<double *>(scratch + (size_t)NA_MAX_POINTS * 4);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = (n_point + NA_THREADS - 1) / NA_THREADS;
    if (low_dim == 2) {
        k_na_pairs<2><<<nb, NA_THREADS, 0, st>>>(n_point, Y, g, zpart);
        k_na_force<2><<<nb, NA_THREADS, 0, st>>>(n_point, nb, g, zpart, F, Z);
    } else {
        k_na_pairs<3><<<nb, NA_THREADS, 0, st>>>(n_point, Y, g, zpart);
        k_na_force<3><<<nb, NA_THREADS, 0, st>>>(n_point, nb, g, zpart, F, Z);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "tsne_exact_repulsion_static: launch failed: %s\n", cudaGetErrorString(e));
        return -2;
    }
    return 0;
}
