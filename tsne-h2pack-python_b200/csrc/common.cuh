// Shared definitions of the B200 t-SNE engine: error handling, per-dimension vector
// types, warp helpers and the design constants of the H2 matrix.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#define TSNE_CUDA_CHECK(expr)                                                              \
    do {                                                                                   \
        cudaError_t err_ = (expr);                                                         \
        if (err_ != cudaSuccess) {                                                         \
            fprintf(stderr, "tsne_h2pack: CUDA error %s at %s:%d: %s\n",                  \
                    cudaGetErrorName(err_), __FILE__, __LINE__, cudaGetErrorString(err_)); \
            throw tsne::CudaError(err_);                                                   \
        }                                                                                  \
    } while (0)

namespace tsne {

struct CudaError {
    cudaError_t code;
    explicit CudaError(cudaError_t c) : code(c) {}
};

// ---------------------------------------------------------------------------------
// H2 design constants (the CPU oracle defines the same values; a unit test compares)
// ---------------------------------------------------------------------------------
constexpr int KEY_DEPTH_2D = 24;          // tree depth limit = Morton bits per dimension
constexpr int KEY_DEPTH_3D = 20;
constexpr double MIN_HALF_WIDTH = 5e-5;   // root half-width = this * 2^k
constexpr int MIN_ADM_LEVEL = 2;          // first level that can hold admissible pairs
constexpr double ID_TOL_FACTOR = 0.1;     // the ID stops at this fraction of h2_tol
constexpr int MAX_RANK_2D = 64;
constexpr int MAX_RANK_3D = 64;
constexpr int N_SHELL = 4;                // proxy shells |y - c|_inf = rho * h
__host__ __device__ constexpr double shell_rho(int k)
{
    return k == 0 ? 3.0 : k == 1 ? 4.5 : k == 2 ? 7.0 : 12.0;
}
constexpr int SHELL_PTS_2D = 16;          // points per square shell
constexpr int SHELL_GRID_3D = 3;          // g x g points per cube face
constexpr int ADM_EXTRA = 2;              // admissible: dist >= w_t + w_s + ADM_EXTRA * min(w)
// Per-node capacity of the inadmissible-source sets carried down the tree
constexpr int NSET_CAP_2D = 48;
constexpr int NSET_CAP_3D = 160;

template <int D> struct Dim;
template <> struct Dim<2> {
    using vec = float2;
    static constexpr int L = KEY_DEPTH_2D;
    static constexpr int MAXR = MAX_RANK_2D;
    static constexpr int NPROXY = N_SHELL * SHELL_PTS_2D;
    static constexpr int NSET = NSET_CAP_2D;
};
template <> struct Dim<3> {
    using vec = float4;   // w unused: one 16-byte load per point
    static constexpr int L = KEY_DEPTH_3D;
    static constexpr int MAXR = MAX_RANK_3D;
    static constexpr int NPROXY = N_SHELL * 6 * SHELL_GRID_3D * SHELL_GRID_3D;
    static constexpr int NSET = NSET_CAP_3D;
};

__device__ __forceinline__ float vget(const float2 &v, int k) { return k == 0 ? v.x : v.y; }
__device__ __forceinline__ float vget(const float4 &v, int k)
{
    return k == 0 ? v.x : (k == 1 ? v.y : v.z);
}
__device__ __forceinline__ void vset(float2 &v, int k, float x) { if (k == 0) v.x = x; else v.y = x; }
__device__ __forceinline__ void vset(float4 &v, int k, float x)
{
    if (k == 0) v.x = x; else if (k == 1) v.y = x; else v.z = x;
}

// squared distance and the repulsive kernel (1 + r^2)^-2
__device__ __forceinline__ float dist2(const float2 &a, const float2 &b)
{
    const float dx = a.x - b.x, dy = a.y - b.y;
    return fmaf(dx, dx, dy * dy);
}
__device__ __forceinline__ float dist2(const float4 &a, const float4 &b)
{
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}
// Hardware reciprocal (PTX rcp.approx, about 1 ulp); the argument is >= 1 here.
__device__ __forceinline__ float fast_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rkernel(float r2)
{
    const float w = fast_rcp(1.0f + r2);
    return w * w;
}

// Packed pairs of floats for the sm_100 paired FP32 instructions (PTX add/sub/mul/fma .f32x2):
// one instruction applies the operation to both halves, halving the issue slots of
// arithmetic that runs on two independent lanes of data (here: two target points).
struct F2 {
    unsigned long long v;
};
__device__ __forceinline__ F2 f2_pack(float lo, float hi)
{
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(F2 a, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ F2 f2_sub(F2 a, F2 b)
{
    F2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 f2_add(F2 a, F2 b)
{
    F2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b)
{
    F2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 f2_fma(F2 a, F2 b, F2 c)
{
    F2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}
// (1 + |a - s|^2)^-2 for two targets a (packed x and y) against one source s (each
// coordinate duplicated in both halves)
__device__ __forceinline__ F2 f2_rkernel(F2 ax, F2 ay, F2 sx, F2 sy)
{
    const F2 dx = f2_sub(ax, sx), dy = f2_sub(ay, sy);
    const F2 q = f2_fma(dx, dx, f2_fma(dy, dy, f2_pack(1.f, 1.f)));
    float q0, q1;
    f2_unpack(q, q0, q1);
    const F2 w = f2_pack(fast_rcp(q0), fast_rcp(q1));
    return f2_mul(w, w);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__host__ __device__ inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Fixed launch geometry of the row-parallel kernels: results are reduced block-wise in a
// fixed order, so the grid must not depend on the device's occupancy.
constexpr int ROW_BLOCK = 256;        // 8 warps
constexpr int ROW_GRID = 148 * 8;     // 8 blocks per SM on a 148-SM B200
constexpr int RED_BLOCK = 256;

}  // namespace tsne
