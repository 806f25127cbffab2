// Exact k nearest neighbours with the distance tiles on the tensor cores (tcgen05).
//
// The scan of k_knn_tiled (knn.cu) spends its time on d^2 = |q|^2 + |p|^2 - 2 q.p in FP32 on the
// CUDA cores. Here the dot products of a 128-query x 128-point tile are tcgen05.mma products
// (kind::f16, FP32 accumulation in tensor memory) of a split of the centred, power-of-two-scaled
// coordinates into FP16 high and low parts: q.p = qh.ph + qh.pl + ql.ph + ql.pl, the last term
// (about 2^-22 of the product) dropped, so the products carry about FP32 precision. The points
// are split once into a tile-blocked array in the operands' shared-memory layout (K-major, no
// swizzle: core matrices of 8 rows x 16 bytes, the 8 16-byte chunks of a row's 64 dimensions
// 128 bytes apart, 8-row groups 1024 bytes apart), with the tile's norms behind, so one bulk
// copy brings a tile into shared memory.
//
// One CTA of 160 threads per 128 queries: warp 4 (one thread) loads point tiles (two stages)
// and issues the 12 MMAs of a tile (3 products x 4 K-steps of 16) into one of two 128-column
// accumulators in tensor memory; warps 0-3 (thread = query row = tensor-memory lane) read the
// tile's 128 dot products, form the distances and keep the row's best k in a max-heap ordered
// by (distance, index), as k_knn_tiled's selection keeps them (ties: the smaller index). The
// stages and accumulators are handed over with mbarriers; every wait is bounded (about two
// seconds), after which the kernel records an error the host reports, and once one wait of the
// launch has given up every other wait returns at once. The output rows are
// sorted by index and the reported distances recomputed from the FP32 coordinates' differences.
#include <cuda_fp16.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cmath>

#include "common.cuh"
#include "devbuf.h"

namespace {

constexpr int TC_M = 128;                                  // queries per CTA (MMA M)
constexpr int TC_N = 128;                                  // points per tile (MMA N)
constexpr int TC_K = 64;                                   // dimensions, zero-padded (4 MMA K-steps)
constexpr int TC_HALF_BYTES = TC_M * TC_K * 2;             // one FP16 part of a tile
constexpr int TC_BLOCK = 2 * TC_HALF_BYTES + TC_N * 4;     // high part, low part, norms
constexpr int TC_THREADS = 160;
constexpr int TC_MAX_K = 128;
constexpr int TC_TMEM_COLS = 2 * TC_N;                     // two accumulators
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;   // bound of one wait
static_assert(TC_M == TC_N, "the query tile is a point tile");
static_assert(TC_BLOCK % 16 == 0, "bulk copies move multiples of 16 bytes");

// byte offset of element (row, k) of a tile part in the K-major no-swizzle operand layout
__host__ __device__ constexpr int tc_off(int row, int k)
{
    return ((row >> 3) * (TC_K / 8) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// wait for the phase of parity `parity` to complete; false when the bound ran out (the wait
// then sets *err) or when another wait of the launch already gave up (so that a launch that
// fails stops within about one bound, not one bound per wait)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err)
{
    const unsigned long long t0 = global_ns();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (*reinterpret_cast<volatile int *>(err) != 0) return false;
        if (global_ns() - t0 > TC_WAIT_NS) {
            atomicExch(err, 1);
            return false;
        }
    }
}
// global -> shared bulk copy completing on an mbarrier (16-byte aligned, multiple of 16 bytes)
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t holder, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(holder), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor of a K-major, no-swizzle operand at shared address `addr`:
// start address and the two byte offsets in 16-byte units (leading: the K-adjacent core
// matrix, 128 bytes; stride: the next 8-row group, 1024 bytes), descriptor version 1
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46);
}
// instruction descriptor: FP32 accumulator, FP16 A and B, both K-major, N = 128, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(TC_IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}
// arrive on `bar` once every MMA issued so far by this thread has completed
__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// all 128 columns of the warp's 32 tensor-memory lanes (thread = lane), in one load
__device__ __forceinline__ void tmem_ld128(uint32_t taddr, uint32_t (&v)[128])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x128.b32 {"
        "%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63, "
        "%64, %65, %66, %67, %68, %69, %70, %71, %72, %73, %74, %75, %76, %77, %78, %79, "
        "%80, %81, %82, %83, %84, %85, %86, %87, %88, %89, %90, %91, %92, %93, %94, %95, "
        "%96, %97, %98, %99, %100, %101, %102, %103, %104, %105, %106, %107, %108, %109, %110, %111, "
        "%112, %113, %114, %115, %116, %117, %118, %119, %120, %121, %122, %123, %124, %125, %126, %127"
        "}, [%128];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]),
          "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]),
          "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
          "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]),
          "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63]),
          "=r"(v[64]), "=r"(v[65]), "=r"(v[66]), "=r"(v[67]), "=r"(v[68]), "=r"(v[69]), "=r"(v[70]), "=r"(v[71]),
          "=r"(v[72]), "=r"(v[73]), "=r"(v[74]), "=r"(v[75]), "=r"(v[76]), "=r"(v[77]), "=r"(v[78]), "=r"(v[79]),
          "=r"(v[80]), "=r"(v[81]), "=r"(v[82]), "=r"(v[83]), "=r"(v[84]), "=r"(v[85]), "=r"(v[86]), "=r"(v[87]),
          "=r"(v[88]), "=r"(v[89]), "=r"(v[90]), "=r"(v[91]), "=r"(v[92]), "=r"(v[93]), "=r"(v[94]), "=r"(v[95]),
          "=r"(v[96]), "=r"(v[97]), "=r"(v[98]), "=r"(v[99]), "=r"(v[100]), "=r"(v[101]), "=r"(v[102]), "=r"(v[103]),
          "=r"(v[104]), "=r"(v[105]), "=r"(v[106]), "=r"(v[107]), "=r"(v[108]), "=r"(v[109]), "=r"(v[110]), "=r"(v[111]),
          "=r"(v[112]), "=r"(v[113]), "=r"(v[114]), "=r"(v[115]), "=r"(v[116]), "=r"(v[117]), "=r"(v[118]), "=r"(v[119]),
          "=r"(v[120]), "=r"(v[121]), "=r"(v[122]), "=r"(v[123]), "=r"(v[124]), "=r"(v[125]), "=r"(v[126]), "=r"(v[127])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// The tile-blocked FP16 split of the centred coordinates (n x dp, row-major) scaled by `scale`
// (a power of two, so the split is exact to FP16 rounding), and each point's squared norm of the
// scaled FP32 coordinates. Points n .. ntile * 128 - 1 and dimensions dim .. 63 are zero.
__global__ void k_tc_split(int n, int n_pad, int dp, int dim, float scale, const float *__restrict__ X,
                           unsigned char *__restrict__ blocks)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    unsigned char *blk = blocks + (size_t)(i / TC_N) * TC_BLOCK;
    const int row = i % TC_N;
    float s2 = 0.f;
    for (int k = 0; k < TC_K; k++) {
        const float v = (i < n && k < dim) ? X[(size_t)i * dp + k] * scale : 0.f;
        const __half h = __float2half_rn(v);
        const __half l = __float2half_rn(v - __half2float(h));
        *reinterpret_cast<__half *>(blk + tc_off(row, k)) = h;
        *reinterpret_cast<__half *>(blk + TC_HALF_BYTES + tc_off(row, k)) = l;
        s2 = fmaf(v, v, s2);
    }
    reinterpret_cast<float *>(blk + 2 * TC_HALF_BYTES)[row] = s2;
}

struct TcBars {
    uint32_t a, full[2], empty[2], acc_full[2], acc_empty[2];
};

// warp 4, one thread: the query tile, then per point tile u (tiles taken from the CTA's own
// tile on, wrapping around): load u + 1 into the other stage once the MMAs of u - 1 released it,
// wait for u's stage and for the epilogue to have released u's accumulator (tile u - 2), issue
// the 12 MMAs, commit to the accumulator's and the stage's barriers
__device__ bool tc_producer(const unsigned char *blocks, int qt, int ntile, uint32_t sA, uint32_t sB, uint32_t tmem,
                            const TcBars &b, int *err)
{
    bool ok = true;
    mbar_expect_tx(b.a, TC_BLOCK);
    bulk_copy(sA, blocks + (size_t)qt * TC_BLOCK, TC_BLOCK, b.a);
    auto load = [&](int u) {
        const int s = u & 1;
        mbar_expect_tx(b.full[s], TC_BLOCK);
        bulk_copy(sB + s * TC_BLOCK, blocks + (size_t)((qt + u) % ntile) * TC_BLOCK, TC_BLOCK, b.full[s]);
    };
    load(0);
    ok &= mbar_wait(b.a, 0, err);
    for (int u = 0; u < ntile; u++) {
        if (u + 1 < ntile) {
            if (u + 1 >= 2) ok &= mbar_wait(b.empty[(u + 1) & 1], (((u + 1) >> 1) - 1) & 1, err);
            load(u + 1);
        }
        const int s = u & 1;
        ok &= mbar_wait(b.full[s], (u >> 1) & 1, err);
        if (u >= 2) ok &= mbar_wait(b.acc_empty[s], ((u >> 1) - 1) & 1, err);
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(s * TC_N);
        const uint32_t bs = sB + s * TC_BLOCK;
        for (int ks = 0; ks < TC_K / 16; ks++) {
            const uint32_t ko = ks * 256;   // two 16-byte K chunks per step
            tc_mma(d, tc_desc(sA + ko), tc_desc(bs + ko), ks > 0);
            tc_mma(d, tc_desc(sA + ko), tc_desc(bs + TC_HALF_BYTES + ko), 1);
            tc_mma(d, tc_desc(sA + TC_HALF_BYTES + ko), tc_desc(bs + ko), 1);
        }
        tc_commit(b.acc_full[s]);
        tc_commit(b.empty[s]);
    }
    // the last commits: every MMA has finished before the CTA frees tensor memory
    if (ntile >= 1) ok &= mbar_wait(b.empty[(ntile - 1) & 1], ((ntile - 1) >> 1) & 1, err);
    return ok;
}

// max-heap of the row's best kh candidates (root: the worst, by (distance, index)) in shared
// memory, position e of row r at e * TC_M + r; replace the root with (d, p) and sift down
__device__ __forceinline__ void heap_sift(float *hd, int *hx, int kh, int r, float d, int p)
{
    int pos = 0;
    for (;;) {
        int c = 2 * pos + 1;
        if (c >= kh) break;
        float dc = hd[c * TC_M + r];
        int ic = hx[c * TC_M + r];
        if (c + 1 < kh) {
            const float d2 = hd[(c + 1) * TC_M + r];
            const int i2 = hx[(c + 1) * TC_M + r];
            if (d2 > dc || (d2 == dc && i2 > ic)) { c++; dc = d2; ic = i2; }
        }
        if (!(dc > d || (dc == d && ic > p))) break;
        hd[pos * TC_M + r] = dc;
        hx[pos * TC_M + r] = ic;
        pos = c;
    }
    hd[pos * TC_M + r] = d;
    hx[pos * TC_M + r] = p;
}
__device__ __noinline__ void heap_replace(float *hd, int *hx, int kh, int r, float d, int p)
{
    heap_sift(hd, hx, kh, r, d, p);
}

// element b (a runtime index below 32) of the registers v[base .. base + 31]: a tree of selects,
// so the array stays in registers
template <int N>
__device__ __forceinline__ float pick32(const uint32_t (&v)[N], int base, int b)
{
    float x[16];
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = __uint_as_float((b & 16) ? v[base + 16 + i] : v[base + i]);
#pragma unroll
    for (int w = 8; w >= 1; w >>= 1) {
#pragma unroll
        for (int i = 0; i < w; i++) x[i] = (b & w) ? x[w + i] : x[i];
    }
    return x[0];
}

// warps 0-3: thread r = query q0 + r = tensor-memory lane r. Per tile: the tile's norms (thread
// r loads column r's, one tile ahead, exchanged through shared memory), the 128 dot products in
// one tensor-memory load (the accumulator is released as soon as they are in registers), the
// distances and their minimum per 32-column chunk; in a chunk whose minimum reaches the row's
// threshold the candidates form a bit mask, and only its set bits are tested again and inserted
__device__ bool tc_epilogue(int n, int kh, int qt, int ntile, const unsigned char *blocks, const float *qnorm,
                            uint32_t tmem, const TcBars &b, float *hd, int *hx, float *nbuf, int *err)
{
    bool ok = true;
    const int r = threadIdx.x, wid = r >> 5;
    const int q = qt * TC_M + r;
    const bool live = q < n;
    auto norm_at = [&](int u) {
        const int ti = (qt + u) % ntile;
        return __ldg(reinterpret_cast<const float *>(blocks + (size_t)ti * TC_BLOCK + 2 * TC_HALF_BYTES) + r);
    };
    ok &= mbar_wait(b.a, 0, err);
    const float qn = qnorm[r];
    float tau = INFINITY;
    int taui = INT_MAX;
    float pn_next = norm_at(0);
    for (int u = 0; u < ntile; u++) {
        const int s = u & 1;
        const int p0 = ((qt + u) % ntile) * TC_N;
        nbuf[s * TC_N + r] = pn_next;
        if (u + 1 < ntile) pn_next = norm_at(u + 1);
        asm volatile("bar.sync 1, %0;" ::"n"(TC_M) : "memory");
        ok &= mbar_wait(b.acc_full[s], (u >> 1) & 1, err);
        tc_fence_after();
        uint32_t v[TC_N];
        tmem_ld128(tmem + ((uint32_t)(wid * 32) << 16) + (uint32_t)(s * TC_N), v);
        tc_fence_before();
        mbar_arrive(b.acc_empty[s]);
        const float *nb = nbuf + s * TC_N;
        float cmin[TC_N / 32] = {INFINITY, INFINITY, INFINITY, INFINITY};   // per 32-column chunk
#pragma unroll
        for (int j = 0; j < TC_N; j++) {
            const float d = fmaxf(fmaf(-2.f, __uint_as_float(v[j]), qn + nb[j]), 0.f);
            v[j] = __float_as_uint(d);
            cmin[j >> 5] = fminf(cmin[j >> 5], d);
        }
        if (!live) continue;
#pragma unroll
        for (int c = 0; c < TC_N / 32; c++) {
            if (!(cmin[c] <= tau)) continue;
            // the chunk's candidates as a bit mask (no branches), then only its set bits
            uint32_t mask = 0;
#pragma unroll
            for (int b = 0; b < 32; b++) {
                const float d = __uint_as_float(v[32 * c + b]);
                const int p = p0 + 32 * c + b;
                const bool pass = (d < tau || (d == tau && p < taui)) && p < n && p != q;
                mask |= (uint32_t)pass << b;
            }
            while (mask != 0) {
                const int b = __ffs(mask) - 1;
                mask &= mask - 1;
                const float d = pick32(v, 32 * c, b);
                const int p = p0 + 32 * c + b;
                if (d < tau || (d == tau && p < taui)) {
                    heap_replace(hd, hx, kh, r, d, p);
                    tau = hd[r];
                    taui = hx[r];
                }
            }
        }
    }
    return ok;
}

constexpr int TC_MARGIN = 16;   // candidates kept beyond k, re-ranked by exact distances

int tc_heap_size(int k) { return std::min(k + TC_MARGIN, TC_MAX_K); }

size_t tc_smem_bytes(int kh)
{
    return (size_t)3 * TC_BLOCK + (size_t)kh * TC_M * (sizeof(float) + sizeof(int)) + 2 * TC_N * sizeof(float) +
           16 * sizeof(uint64_t);
}

__global__ void __launch_bounds__(TC_THREADS, 1)
k_knn_tc(int n, int dp, int k, int kh, int ntile, const unsigned char *__restrict__ blocks,
         const float *__restrict__ X, int *__restrict__ out_idx, float *__restrict__ out_d, int *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    unsigned char *sA = sm, *sB = sm + TC_BLOCK;
    float *hd = reinterpret_cast<float *>(sm + 3 * TC_BLOCK);
    int *hx = reinterpret_cast<int *>(hd + (size_t)kh * TC_M);
    float *nbuf = reinterpret_cast<float *>(hx + (size_t)kh * TC_M);
    uint64_t *bars = reinterpret_cast<uint64_t *>(nbuf + 2 * TC_N);
    uint32_t *holder = reinterpret_cast<uint32_t *>(bars + 9);
    TcBars b;
    b.a = smem_u32(bars);
    for (int s = 0; s < 2; s++) {
        b.full[s] = smem_u32(bars + 1 + s);
        b.empty[s] = smem_u32(bars + 3 + s);
        b.acc_full[s] = smem_u32(bars + 5 + s);
        b.acc_empty[s] = smem_u32(bars + 7 + s);
    }
    const int qt = blockIdx.x;
    if (wid == 4) {
        tmem_alloc(smem_u32(holder), TC_TMEM_COLS);
        tmem_relinquish();
        if (lane == 0) {
            mbar_init(b.a, 1);
            for (int s = 0; s < 2; s++) {
                mbar_init(b.full[s], 1);
                mbar_init(b.empty[s], 1);
                mbar_init(b.acc_full[s], 1);
                mbar_init(b.acc_empty[s], TC_M);
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    } else {
        for (int e = 0; e < kh; e++) {
            hd[e * TC_M + tid] = INFINITY;
            hx[e * TC_M + tid] = INT_MAX;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *holder;
    bool ok = true;
    if (wid == 4) {
        if (lane == 0) ok = tc_producer(blocks, qt, ntile, smem_u32(sA), smem_u32(sB), tmem, b, err);
    } else {
        ok = tc_epilogue(n, kh, qt, ntile, blocks, reinterpret_cast<const float *>(sA + 2 * TC_HALF_BYTES), tmem, b,
                         hd, hx, nbuf, err);
    }
    if (!ok) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    if (wid == 4) {
        tc_fence_after();
        tmem_dealloc(tmem, TC_TMEM_COLS);
        return;
    }
    // the kh candidates' distances from the FP32 coordinates' differences; the k best of them by
    // (distance, index), reported in index order
    const int q = qt * TC_M + tid;
    if (q >= n) return;
    const float *xq = X + (size_t)q * dp;
    for (int t = 0; t < kh; t++) {
        const int j = hx[t * TC_M + tid];
        float d2 = INFINITY;
        if (j >= 0 && j < n) {
            const float *xj = X + (size_t)j * dp;
            d2 = 0.f;
            for (int c = 0; c < dp; c += 4) {
                const float4 a4 = *reinterpret_cast<const float4 *>(xq + c);
                const float4 b4 = *reinterpret_cast<const float4 *>(xj + c);
                const float dx = a4.x - b4.x, dy = a4.y - b4.y, dz = a4.z - b4.z, dw = a4.w - b4.w;
                d2 = fmaf(dx, dx, d2); d2 = fmaf(dy, dy, d2); d2 = fmaf(dz, dz, d2); d2 = fmaf(dw, dw, d2);
            }
        }
        hd[t * TC_M + tid] = d2;
    }
    for (int a = 1; a < kh; a++) {   // by (distance, index)
        const float da = hd[a * TC_M + tid];
        const int ia = hx[a * TC_M + tid];
        int z = a - 1;
        while (z >= 0 && (hd[z * TC_M + tid] > da || (hd[z * TC_M + tid] == da && hx[z * TC_M + tid] > ia))) {
            hd[(z + 1) * TC_M + tid] = hd[z * TC_M + tid];
            hx[(z + 1) * TC_M + tid] = hx[z * TC_M + tid];
            z--;
        }
        hd[(z + 1) * TC_M + tid] = da;
        hx[(z + 1) * TC_M + tid] = ia;
    }
    for (int a = 1; a < k; a++) {    // the first k by index
        const float da = hd[a * TC_M + tid];
        const int ia = hx[a * TC_M + tid];
        int z = a - 1;
        while (z >= 0 && hx[z * TC_M + tid] > ia) {
            hd[(z + 1) * TC_M + tid] = hd[z * TC_M + tid];
            hx[(z + 1) * TC_M + tid] = hx[z * TC_M + tid];
            z--;
        }
        hd[(z + 1) * TC_M + tid] = da;
        hx[(z + 1) * TC_M + tid] = ia;
    }
    for (int t = 0; t < k; t++) {
        out_idx[(size_t)q * k + t] = hx[t * TC_M + tid];
        out_d[(size_t)q * k + t] = sqrtf(hd[t * TC_M + tid]);
    }
}

}  // namespace

namespace tsne {

// The tensor-core scan for k <= 128 neighbours of points with at most 64 (centred) dimensions:
// dX is n x dp (dp a multiple of 4) on the device, maxabs its largest absolute coordinate;
// indices and distances (n x k, rows sorted by index) to dI / dD. 0 done, 1 not applicable
// (the caller takes the CUDA-core scan), -1 a bounded wait gave up.
int knn_tc_run(const float *dX, int n, int dp, int dim, int k, float maxabs, int *dI, float *dD, cudaStream_t st)
{
    if (dim > TC_K || k > TC_MAX_K || k < 1 || n < 2) return 1;
    const char *e = getenv("TSNE_KNN_TC");
    if (e != nullptr && atoi(e) == 0) return 1;
    const int ntile = (n + TC_N - 1) / TC_N;
    // scale by a power of two so that the largest coordinate lies in [256, 512): far from the
    // FP16 range's ends, and the split stays exact to FP16 rounding
    float scale = 1.f;
    if (maxabs > 0.f && std::isfinite(maxabs)) scale = std::ldexp(1.f, (int)std::floor(std::log2(256.f / maxabs)) + 1);
    while (maxabs * scale >= 512.f) scale *= 0.5f;
    DevBuf<unsigned char> blocks;
    DevBuf<int> err;
    blocks.exact((size_t)ntile * TC_BLOCK);
    err.exact(1);
    TSNE_CUDA_CHECK(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    k_tc_split<<<(ntile * TC_N + 255) / 256, 256, 0, st>>>(n, ntile * TC_N, dp, dim, scale, dX, blocks.p);
    const int kh = tc_heap_size(k);
    const size_t smem = tc_smem_bytes(kh);
    TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_knn_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_knn_tc<<<ntile, TC_THREADS, smem, st>>>(n, dp, k, kh, ntile, blocks.p, dX, dI, dD, err.p);
    TSNE_CUDA_CHECK(cudaGetLastError());
    int herr = 0;
    TSNE_CUDA_CHECK(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    if (herr) fprintf(stderr, "tsne_h2pack: the tensor-core k-NN scan's bounded wait gave up\n");
    return herr ? -1 : 0;
}

}  // namespace tsne
