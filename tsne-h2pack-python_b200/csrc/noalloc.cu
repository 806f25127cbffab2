// tsne_exact_repulsion_static: the exact O(N^2) repulsive force for callers that cannot
// allocate device memory.
//
// Some callers must not allocate: code that runs under a caller-owned memory budget (a
// serving process that has carved HBM up front and may not grow), code that runs inside a
// region where an allocation's implicit device synchronisation is not acceptable, or hosts
// whose allocator is not the CUDA runtime's. This entry point takes device pointers for its
// input and outputs and keeps its scratch (the sums s and v and the Z partials) in a
// file-scope __device__ array of fixed size, so it calls no cudaMalloc, cudaFree or any other
// allocating routine.
//
// The scratch array exists once per device and is shared by every call on that device: calls
// that overlap on the GPU (two streams at once, or two host threads) race on it. Every
// element a call reads is written earlier by the same call, so no clearing is needed.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "common.cuh"
#include "../../include/tsne_h2pack.h"

namespace {

using namespace tsne;

constexpr int NA_MAX_POINTS = 65536;                       // largest n_point accepted
constexpr int NA_BLOCKS = 148 * 2;                         // Z partial blocks (fixed order)
constexpr size_t NA_SCRATCH_FLOATS = (size_t)NA_MAX_POINTS * 4 + (size_t)NA_BLOCKS * 3 * 2;

// s (n floats), v (3 n floats), then NA_BLOCKS x 3 doubles of Z partials
static __device__ __align__(256) float na_scratch[NA_SCRATCH_FLOATS];

constexpr int NA_MAX_DEVICES = 64;
float *na_ptr[NA_MAX_DEVICES] = {nullptr};

template <int D>
__device__ __forceinline__ void load_pt(const float *Y, int i, float (&p)[D])
{
#pragma unroll
    for (int k = 0; k < D; k++) p[k] = Y[(size_t)i * D + k];
}

// s_i = sum_{j != i} K_ij, v_i = sum_{j != i} K_ij y_j (the exact path of the engine,
// reading point-major coordinates); sources staged 256 at a time in shared memory
template <int D>
__global__ void __launch_bounds__(256) k_na_sv(int n, const float *__restrict__ Y, float *__restrict__ scratch)
{
    __shared__ float sh[256][D];
    const int i = blockIdx.x * 256 + threadIdx.x;
    float yi[D];
    for (int k = 0; k < D; k++) yi[k] = 0.f;
    if (i < n) load_pt<D>(Y, i, yi);
    double S = 0.0, V[D];
    for (int k = 0; k < D; k++) V[k] = 0.0;
    for (int base = 0; base < n; base += 256) {
        __syncthreads();
        if (base + (int)threadIdx.x < n)
            for (int k = 0; k < D; k++) sh[threadIdx.x][k] = Y[(size_t)(base + threadIdx.x) * D + k];
        __syncthreads();
        const int cnt = min(256, n - base);
        float ts = 0.f, tv[D];
        for (int k = 0; k < D; k++) tv[k] = 0.f;
        for (int j = 0; j < cnt; j++) {
            float r2 = 0.f;
#pragma unroll
            for (int k = 0; k < D; k++) { const float df = yi[k] - sh[j][k]; r2 = fmaf(df, df, r2); }
            float w = rkernel(r2);
            w = (base + j == i) ? 0.f : w;
            ts += w;
#pragma unroll
            for (int k = 0; k < D; k++) tv[k] = fmaf(w, sh[j][k], tv[k]);
        }
        S += ts;
        for (int k = 0; k < D; k++) V[k] += tv[k];
    }
    if (i < n) {
        scratch[i] = (float)S;
        for (int k = 0; k < D; k++) scratch[(size_t)NA_MAX_POINTS + (size_t)i * 3 + k] = (float)V[k];
    }
}

// Z = sum s + 2 sum |y|^2 s - 2 sum y.v, partial sums per block (fixed grid)
template <int D>
__global__ void __launch_bounds__(256) k_na_zpart(int n, const float *__restrict__ Y, float *__restrict__ scratch)
{
    double t[3] = {0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double s = scratch[i];
        double yy = 0.0, yv = 0.0;
        for (int k = 0; k < D; k++) {
            const double y = Y[(size_t)i * D + k];
            yy += y * y;
            yv += y * (double)scratch[(size_t)NA_MAX_POINTS + (size_t)i * 3 + k];
        }
        t[0] += s; t[1] += yy * s; t[2] += yv;
    }
    __shared__ double sh[256][3];
    for (int k = 0; k < 3; k++) sh[threadIdx.x][k] = t[k];
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int k = 0; k < 3; k++) sh[threadIdx.x][k] += sh[threadIdx.x + st][k];
        __syncthreads();
    }
    double *part = reinterpret_cast<double *>(scratch + (size_t)NA_MAX_POINTS * 4);
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; k++) part[(size_t)blockIdx.x * 3 + k] = sh[0][k];
}

// F_i = (4 / Z)(y_i s_i - v_i); every block sums the partials in the same order
template <int D>
__global__ void __launch_bounds__(256) k_na_force(int n, const float *__restrict__ Y, const float *__restrict__ scratch,
                                                  float *__restrict__ F, double *__restrict__ Zout)
{
    __shared__ double sh[256][3];
    const double *part = reinterpret_cast<const double *>(scratch + (size_t)NA_MAX_POINTS * 4);
    double t[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < NA_BLOCKS; b += blockDim.x)
        for (int k = 0; k < 3; k++) t[k] += part[(size_t)b * 3 + k];
    for (int k = 0; k < 3; k++) sh[threadIdx.x][k] = t[k];
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int k = 0; k < 3; k++) sh[threadIdx.x][k] += sh[threadIdx.x + st][k];
        __syncthreads();
    }
    const double Z = sh[0][0] + 2.0 * sh[0][1] - 2.0 * sh[0][2];
    if (blockIdx.x == 0 && threadIdx.x == 0) *Zout = Z;
    const double c = 4.0 / Z;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double s = scratch[i];
        for (int k = 0; k < D; k++) {
            const double y = Y[(size_t)i * D + k];
            const double v = scratch[(size_t)NA_MAX_POINTS + (size_t)i * 3 + k];
            F[(size_t)i * D + k] = (float)(c * (y * s - v));
        }
    }
}

// Device address of the scratch array on the current device, looked up once per device.
float *scratch_address(int *err)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) { *err = -2; return nullptr; }
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
    int err = 0;
    float *scratch = scratch_address(&err);
    if (scratch == nullptr) return err;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = (n_point + 255) / 256;
    if (low_dim == 2) {
        k_na_sv<2><<<nb, 256, 0, st>>>(n_point, Y, scratch);
        k_na_zpart<2><<<NA_BLOCKS, 256, 0, st>>>(n_point, Y, scratch);
        k_na_force<2><<<nb, 256, 0, st>>>(n_point, Y, scratch, F, Z);
    } else {
        k_na_sv<3><<<nb, 256, 0, st>>>(n_point, Y, scratch);
        k_na_zpart<3><<<NA_BLOCKS, 256, 0, st>>>(n_point, Y, scratch);
        k_na_force<3><<<nb, 256, 0, st>>>(n_point, Y, scratch, F, Z);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "tsne_exact_repulsion_static: launch failed: %s\n", cudaGetErrorString(e));
        return -2;
    }
    return 0;
}
