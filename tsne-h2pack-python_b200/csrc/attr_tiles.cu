// The 2D attractive pass over row tiles with shared columns (reference counterpart: the
// attractive sums of src/tsne_attr_2d.h:22-67 and the update of src/tsne_h2pack.c:1942-1968).
//
// Why: the CSR pass (k_attr_update) gathers Y[j] once per P entry, and those scattered 8-byte
// gathers, one L1 sector lookup each, set its time, not HBM. After the renumbering in tree
// order, the 64 consecutive rows of a tile share most of their neighbours: late in a 1M-point
// run a tile holds about 0.63 distinct columns per entry, and 0.45 distinct 32-byte sectors
// (measured on the benchmark's embedding). So each tile's distinct columns are gathered once,
// in sorted order (neighbouring columns share sectors), into shared memory, and the entries
// read Y from there through 16-bit tile-local indices stored beside the values.
//
// Format (built on the device after each renumbering, rows unchanged): for tile t (rows
// R t .. R t + R - 1) the sorted distinct columns ucol[uptr[t] .. uptr[t + 1]); for every
// padded P entry its index into its tile's list (lidx, uint16). Tiles with more than umax
// distinct columns (too many for the shared-memory stage) read Y[col] directly. The stage is
// filled with asynchronous 8-byte copies (cp.async), all of a thread's gathers in flight at once.
//
// The kernel keeps k_attr_update's arithmetic exactly: a row per half-warp, lane l of the half
// summing entries b + 4 l + 64 s in the same order, the same 16-lane reduction and the same
// update, so every row's sums and update are the same bits. Rows are dealt by tiles to a fixed
// grid of persistent CTAs; the centring partials are per CTA (the other ROW_GRID slots zero),
// so the mean is a fixed-order sum, though in another order than the CSR pass's.
#include <cuda_runtime.h>
#include <stdio.h>

#include <algorithm>

#include <cub/cub.cuh>

#include "attr_tiles.h"
#include "common.cuh"
#include "devbuf.h"

namespace tsne {

namespace {

constexpr int TILE_THREADS = 256;           // 16 half-warps, rows / 16 rows each per tile
constexpr int TILE_GRID = 148 * 4;          // persistent CTAs: at most four per SM (registers)
constexpr int TILE_UMAX_CAP = 12288;        // largest shared-memory stage (96 KB)
static_assert(TILE_GRID <= ROW_GRID, "the centring reads ROW_GRID partial slots");

enum { T_FUSED = 0, T_GRAD = 1 };

// 8-byte asynchronous copy global -> shared (the gathers of a tile's stage all in flight)
__device__ __forceinline__ void cp_async8(float2 *dst, const float2 *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void acc_pair(const float2 &yi, const float2 &yj, float p, float (&a)[2])
{
    const float dx = yi.x - yj.x, dy = yi.y - yj.y;
    float r2 = fmaf(dx, dx, 0.f);
    r2 = fmaf(dy, dy, r2);
    const float q = p * fast_rcp(1.0f + r2);
    a[0] = fmaf(q, dx, a[0]);
    a[1] = fmaf(q, dy, a[1]);
}

template <int MODE>
__global__ void __launch_bounds__(TILE_THREADS, 4)
k_attr_tile(int n, int ntile, int rows, int umax, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
            const unsigned short *__restrict__ lidx, const int *__restrict__ uptr, const int *__restrict__ ucol,
            const float2 *__restrict__ Y, float2 *__restrict__ Yn, float2 *__restrict__ uY,
            float2 *__restrict__ gains, const float2 *__restrict__ rep, const int *__restrict__ rep_flag,
            float exag4, float mom, float lr, double *__restrict__ partials, float2 *__restrict__ attr)
{
    extern __shared__ float2 sy[];
    __shared__ double wsum[TILE_THREADS / 32][2];
    const int tid = threadIdx.x, lane = tid & 31, hl = lane & 15, hw = tid >> 4;
    const int use_rep = (MODE == T_FUSED && rep != nullptr) ? *rep_flag : 0;
    double acc[2] = {0.0, 0.0};
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
        const int u0 = uptr[t], u = uptr[t + 1] - u0;
        const bool staged = u <= umax;        // uniform over the CTA
        __syncthreads();                      // the previous tile's reads are done
        if (staged) {
            // column indices eight at a time, then their eight gathers issued without waiting
            for (int k0 = tid; k0 < u; k0 += TILE_THREADS * 8) {
                int c[8];
#pragma unroll
                for (int g = 0; g < 8; g++) {
                    const int k = k0 + g * TILE_THREADS;
                    c[g] = k < u ? __ldg(ucol + u0 + k) : 0;
                }
#pragma unroll
                for (int g = 0; g < 8; g++) {
                    const int k = k0 + g * TILE_THREADS;
                    if (k < u) cp_async8(sy + k, Y + c[g]);
                }
            }
            cp_async_wait_all();
        }
        __syncthreads();
        // every half-warp takes rows / 16 rows, so both halves of a warp run the same rounds
        for (int rr = hw; rr < rows; rr += TILE_THREADS / 16) {
            const int i = t * rows + rr;
            const bool live = i < n;
            float2 yi = make_float2(0.f, 0.f), opnd = make_float2(0.f, 0.f);
            int b = 0, e = 0;
            if (live) {
                yi = Y[i];
                b = rp[i];
                e = rp[i + 1];
                if (MODE == T_FUSED) {
                    if (hl == 1) opnd = uY[i];
                    else if (hl == 2) opnd = gains[i];
                    else if (hl == 3 && use_rep) opnd = rep[i];
                }
            }
            float a[2] = {0.f, 0.f};
            if (staged) {
                for (int base = b + 4 * hl; base < e; base += 64) {
                    const uint2 l4 = __ldcs(reinterpret_cast<const uint2 *>(lidx + base));
                    const float4 p4 = __ldcs(reinterpret_cast<const float4 *>(val + base));
                    acc_pair(yi, sy[l4.x & 0xffffu], p4.x, a);
                    acc_pair(yi, sy[l4.x >> 16], p4.y, a);
                    acc_pair(yi, sy[l4.y & 0xffffu], p4.z, a);
                    acc_pair(yi, sy[l4.y >> 16], p4.w, a);
                }
            } else {
                for (int base = b + 4 * hl; base < e; base += 64) {
                    const int4 c4 = __ldcs(reinterpret_cast<const int4 *>(col + base));
                    const float4 p4 = __ldcs(reinterpret_cast<const float4 *>(val + base));
                    acc_pair(yi, __ldg(Y + c4.x), p4.x, a);
                    acc_pair(yi, __ldg(Y + c4.y), p4.y, a);
                    acc_pair(yi, __ldg(Y + c4.z), p4.z, a);
                    acc_pair(yi, __ldg(Y + c4.w), p4.w, a);
                }
            }
#pragma unroll
            for (int k = 0; k < 2; k++)
                for (int o = 8; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
            if (MODE == T_GRAD) {
                if (live && hl == 0) attr[i] = make_float2(a[0], a[1]);
                continue;
            }
            const int src = lane & 16;
            float2 uu, gg, rr2;
            uu.x = __shfl_sync(0xffffffffu, opnd.x, src + 1);
            uu.y = __shfl_sync(0xffffffffu, opnd.y, src + 1);
            gg.x = __shfl_sync(0xffffffffu, opnd.x, src + 2);
            gg.y = __shfl_sync(0xffffffffu, opnd.y, src + 2);
            rr2.x = __shfl_sync(0xffffffffu, opnd.x, src + 3);
            rr2.y = __shfl_sync(0xffffffffu, opnd.y, src + 3);
            if (live && hl == 0) {
                float2 yn = yi;
                const float uv[2] = {uu.x, uu.y}, gv[2] = {gg.x, gg.y}, rv[2] = {rr2.x, rr2.y}, yv[2] = {yi.x, yi.y};
                float un[2], gn[2], ynv[2];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const float gk = exag4 * a[k] - rv[k];
                    float gain = (uv[k] * gk < 0.f) ? gv[k] + 0.2f : gv[k] * 0.8f;
                    gain = fmaxf(gain, 0.01f);
                    un[k] = mom * uv[k] - lr * (gk * gain);
                    gn[k] = gain;
                    ynv[k] = yv[k] + un[k];
                    acc[k] += (double)ynv[k];
                }
                yn = make_float2(ynv[0], ynv[1]);
                uY[i] = make_float2(un[0], un[1]);
                gains[i] = make_float2(gn[0], gn[1]);
                Yn[i] = yn;
            }
        }
    }
    if (MODE == T_GRAD) return;
    // lanes 0 and 16 of each warp hold partial sums: fold, then warps in order
    for (int k = 0; k < 2; k++) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 16);
    if (lane == 0) { wsum[tid >> 5][0] = acc[0]; wsum[tid >> 5][1] = acc[1]; }
    __syncthreads();
    if (tid == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < TILE_THREADS / 32; w++) { s0 += wsum[w][0]; s1 += wsum[w][1]; }
        partials[(size_t)blockIdx.x * 2] = s0;
        partials[(size_t)blockIdx.x * 2 + 1] = s1;
        for (int b = blockIdx.x + gridDim.x; b < ROW_GRID; b += gridDim.x) {
            partials[(size_t)b * 2] = 0.0;
            partials[(size_t)b * 2 + 1] = 0.0;
        }
    }
}

// ---- format construction ----
__global__ void k_tile_keys(int n, int rows, const int *__restrict__ rp, const int *__restrict__ col,
                            unsigned long long *__restrict__ keys, int *__restrict__ vals)
{
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        const unsigned long long hi = (unsigned long long)(i / rows) << 32;
        for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) {
            keys[e] = hi | (unsigned)col[e];
            vals[e] = e;
        }
    }
}

__global__ void k_tile_heads(long long m, const unsigned long long *__restrict__ keys, int *__restrict__ head)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m; s += (long long)gridDim.x * blockDim.x)
        head[s] = (s == 0 || keys[s] != keys[s - 1]) ? 1 : 0;
}

__global__ void k_tile_ucol(long long m, const unsigned long long *__restrict__ keys, const int *__restrict__ head,
                            const int *__restrict__ pos, int *__restrict__ ucol, int *__restrict__ utile)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m; s += (long long)gridDim.x * blockDim.x) {
        if (!head[s]) continue;
        const unsigned long long k = keys[s];
        ucol[pos[s]] = (int)(k & 0xffffffffULL);
        utile[pos[s]] = (int)(k >> 32);
    }
}

// uptr[t] = first distinct-column slot of tile t (tiles in order; empty tiles repeat)
__global__ void k_tile_uptr(int cnt, int ntile, const int *__restrict__ utile, int *__restrict__ uptr)
{
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u <= cnt; u += (long long)gridDim.x * blockDim.x) {
        const int lo = u == 0 ? -1 : utile[u - 1];
        const int hi = u == cnt ? ntile : utile[u];
        for (int t = lo + 1; t <= hi; t++) uptr[t] = (int)u;
    }
}

__global__ void k_tile_lidx(long long m, const unsigned long long *__restrict__ keys, const int *__restrict__ vals,
                            const int *__restrict__ head, const int *__restrict__ pos, const int *__restrict__ uptr,
                            unsigned short *__restrict__ lidx)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m; s += (long long)gridDim.x * blockDim.x) {
        const int id = pos[s] + head[s] - 1;       // the distinct-column slot of entry s
        const int t = (int)(keys[s] >> 32);
        const int loc = id - uptr[t];
        lidx[vals[s]] = (unsigned short)(loc < 65535 ? loc : 65535);   // tiles that large are not staged
    }
}

int tile_key_bits(int ntile)
{
    int b = 1;
    while ((1 << b) < ntile + 1 && b < 31) b++;
    return 32 + b;
}

}  // namespace

int attr_tiles_build(cudaStream_t st, int n, long long padded_nnz, const int *rp, const int *col, int rows, int umax,
                     AttrTiles &out)
{
    if (padded_nnz + 1 > 0x7fffffffLL || rows < 16 || rows % 16 != 0 || umax < 256 || umax > TILE_UMAX_CAP) return -1;
    const int m = (int)padded_nnz;
    const int ntile = (n + rows - 1) / rows;
    DevBuf<unsigned long long> keys, keys2;
    DevBuf<int> vals, vals2, head, pos;
    keys.exact(std::max(m, 1)); vals.exact(std::max(m, 1));
    k_tile_keys<<<148 * 8, 256, 0, st>>>(n, rows, rp, col, keys.p, vals.p);
    keys2.exact(std::max(m, 1)); vals2.exact(std::max(m, 1));
    {
        size_t bytes = 0;
        TSNE_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.p, keys2.p, vals.p, vals2.p, m, 0,
                                                        tile_key_bits(ntile), st));
        DevBuf<unsigned char> tmp;
        tmp.exact(bytes + 256);
        TSNE_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, keys.p, keys2.p, vals.p, vals2.p, m, 0,
                                                        tile_key_bits(ntile), st));
    }
    keys.release();
    vals.release();
    head.exact((size_t)m + 1);
    pos.exact((size_t)m + 1);
    k_tile_heads<<<148 * 8, 256, 0, st>>>(m, keys2.p, head.p);
    TSNE_CUDA_CHECK(cudaMemsetAsync(head.p + m, 0, sizeof(int), st));
    {
        size_t bytes = 0;
        TSNE_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, head.p, pos.p, m + 1, st));
        DevBuf<unsigned char> tmp;
        tmp.exact(bytes + 256);
        TSNE_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, head.p, pos.p, m + 1, st));
    }
    int cnt = 0;
    TSNE_CUDA_CHECK(cudaMemcpyAsync(&cnt, pos.p + m, sizeof(int), cudaMemcpyDeviceToHost, st));
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    DevBuf<int> utile;
    utile.exact(std::max(cnt, 1));
    out.ucol.exact(std::max(cnt, 1));
    out.uptr.exact((size_t)ntile + 1);
    out.lidx.exact(std::max(m, 4));
    k_tile_ucol<<<148 * 8, 256, 0, st>>>(m, keys2.p, head.p, pos.p, out.ucol.p, utile.p);
    k_tile_uptr<<<148 * 8, 256, 0, st>>>(cnt, ntile, utile.p, out.uptr.p);
    k_tile_lidx<<<148 * 8, 256, 0, st>>>(m, keys2.p, vals2.p, head.p, pos.p, out.uptr.p, out.lidx.p);
    TSNE_CUDA_CHECK(cudaGetLastError());
    out.ntile = ntile;
    out.rows = rows;
    out.umax = umax;
    out.n_unique = cnt;
    out.valid = true;
    return 0;
}

// persistent CTAs resident at once for a stage of umax columns (shared memory per SM 228 KB)
static int tile_grid(int umax)
{
    const int per_sm = std::min(4, (228 * 1024) / (int)(sizeof(float2) * umax + 1024));
    return 148 * std::max(1, per_sm);
}

static void set_smem_once()
{
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev]) return;
    const int smem = (int)(sizeof(float2) * TILE_UMAX_CAP);
    TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_attr_tile<T_FUSED>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_attr_tile<T_GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    done[dev] = true;
}

void launch_attr_tile_update(cudaStream_t st, int n, const AttrTiles &tl, const int *rp, const int *col,
                             const float *val, const void *Y, void *Ynext, void *uY, void *gains, const void *rep,
                             const int *rep_flag, float exag4, float mom, float lr, double *partials)
{
    set_smem_once();
    k_attr_tile<T_FUSED><<<tile_grid(tl.umax), TILE_THREADS, sizeof(float2) * tl.umax, st>>>(
        n, tl.ntile, tl.rows, tl.umax, rp, col, val, tl.lidx.p, tl.uptr.p, tl.ucol.p, (const float2 *)Y, (float2 *)Ynext,
        (float2 *)uY, (float2 *)gains, (const float2 *)rep, rep_flag, exag4, mom, lr, partials, nullptr);
}

void launch_attr_tile_grad(cudaStream_t st, int n, const AttrTiles &tl, const int *rp, const int *col,
                           const float *val, const void *Y, void *attr)
{
    set_smem_once();
    k_attr_tile<T_GRAD><<<tile_grid(tl.umax), TILE_THREADS, sizeof(float2) * tl.umax, st>>>(
        n, tl.ntile, tl.rows, tl.umax, rp, col, val, tl.lidx.p, tl.uptr.p, tl.ucol.p, (const float2 *)Y, nullptr, nullptr, nullptr,
        nullptr, nullptr, 0.f, 0.f, 0.f, nullptr, (float2 *)attr);
}

}  // namespace tsne
