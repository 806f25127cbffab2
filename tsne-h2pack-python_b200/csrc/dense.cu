// Per-point and per-row kernels of the optimisation loop: the attractive CSR pass fused
// with the gains/momentum update, centring, the exact O(N^2) repulsion, the Z identity and
// force assembly, the KL divergence, point renumbering and the perplexity calibration.
//
// Reference counterparts (paths within the reference project):
//   attractive pass ............ src/tsne_attr_2d.h:22-67, src/tsne_h2pack.c:199-356
//   update + centring .......... src/tsne_h2pack.c:1942-1984
//   exact repulsion ............ src/tsne_h2pack.c:404-491
//   Z identity + force ......... src/tsne_h2pack.c:538-627
//   KL ......................... src/tsne_h2pack.c:1870-1895
//   renumbering ................ src/tsne_reorder.c:112-167
//   perplexity calibration ..... src/tsne_utils.c:952-1105
#include <math.h>
#include <stdlib.h>

#include "common.cuh"
#include "kernels.h"

namespace tsne {

namespace {

template <int D> using Vec = typename Dim<D>::vec;

template <int D>
__device__ __forceinline__ Vec<D> vzero()
{
    Vec<D> v;
    if constexpr (D == 2) v = make_float2(0.f, 0.f);
    else v = make_float4(0.f, 0.f, 0.f, 0.f);
    return v;
}

// Streamed P entries: read once per pass, kept out of L1 so Y stays cached.
__device__ __forceinline__ int4 ld_stream_i4(const int *p)
{
    return __ldcs(reinterpret_cast<const int4 *>(p));
}
__device__ __forceinline__ float4 ld_stream_f4(const float *p)
{
    return __ldcs(reinterpret_cast<const float4 *>(p));
}

template <int D>
__device__ __forceinline__ void attr_acc(const Vec<D> &yi, const Vec<D> *__restrict__ Y, int c, float p,
                                         float (&a)[D])
{
    const Vec<D> yj = __ldg(Y + c);
    float df[D], r2 = 0.f;
#pragma unroll
    for (int k = 0; k < D; k++) { df[k] = vget(yi, k) - vget(yj, k); r2 = fmaf(df[k], df[k], r2); }
    const float q = p * fast_rcp(1.0f + r2);
#pragma unroll
    for (int k = 0; k < D; k++) a[k] = fmaf(q, df[k], a[k]);
}

// Warp-per-row attractive sum over a row padded to a multiple of 4 entries; every lane
// reads 4 column indices and 4 values with two 128-bit loads per step.
template <int D>
__device__ __forceinline__ void row_attr(int b, int e, int lane, const Vec<D> &yi, const int *__restrict__ col,
                                         const float *__restrict__ val, const Vec<D> *__restrict__ Y,
                                         float (&a)[D])
{
    for (int base = b + 4 * lane; base < e; base += 128) {
        const int4 c4 = ld_stream_i4(col + base);
        const float4 p4 = ld_stream_f4(val + base);
        attr_acc<D>(yi, Y, c4.x, p4.x, a);
        attr_acc<D>(yi, Y, c4.y, p4.y, a);
        attr_acc<D>(yi, Y, c4.z, p4.z, a);
        attr_acc<D>(yi, Y, c4.w, p4.w, a);
    }
#pragma unroll
    for (int k = 0; k < D; k++) a[k] = warp_sum(a[k]);
}

// Block-wide FP64 reduction of per-warp values held by lane 0 of each warp, summed in
// warp order; the result is valid in thread 0.
template <int NV, int NW = ROW_BLOCK / 32>
__device__ __forceinline__ void block_sum_warps(double (&v)[NV], double *out)
{
    __shared__ double sh[NW][NV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < NV; k++) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; k++) {
            double s = 0.0;
            for (int ww = 0; ww < NW; ww++) s += sh[ww][k];
            out[k] = s;
        }
    }
}

// Fixed-order sum of `count` per-block partials (stride NV) by one block; result in sh_out.
template <int NV>
__device__ __forceinline__ void reduce_partials(const double *__restrict__ part, int count, double *sh_out)
{
    __shared__ double sh[RED_BLOCK][NV];
    double acc[NV];
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < count; b += blockDim.x)
        for (int k = 0; k < NV; k++) acc[k] += part[(size_t)b * NV + k];
    for (int k = 0; k < NV; k++) sh[threadIdx.x][k] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < NV; k++) sh[threadIdx.x][k] += sh[threadIdx.x + s][k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NV; k++) sh_out[k] = sh[0][k];
    __syncthreads();
}

// ---------------------------------------------------------------------------------
// Attractive force + gains / momentum update (reference tsne_h2pack.c:1942-1968):
//   g = 4 exag sum_j p_ij (y_i - y_j) / (1 + |y_i - y_j|^2) - F_rep
//   gain: +0.2 if uY * g < 0 else * 0.8, floor 0.01; uY = mom uY - lr gain g; Y += uY
// Ynext is a separate buffer because other warps still gather the old Y.
// ---------------------------------------------------------------------------------
// Rows are dealt round-robin to half-warps (row i to half-warp i mod H), so that at any
// moment all warps of the device stream one window of P (the HBM traffic stays within a few
// MB of consecutive rows) and every warp has two independent rows, i.e. two streams of P
// loads and Y gathers, in flight. A half-warp reads 64 entries per step (4 per lane, two
// 128-bit loads); lanes 1-3 of the half fetch the row's update operands meanwhile.
// MODE ATTR_FUSED: the whole step. ATTR_GRAD: only the attractive sums, stored in `attr`
// (run while the host reads an H2 build's counts). ATTR_UPDATE: the update from the stored
// sums, with the same rows per thread and the same summation order as ATTR_FUSED, so the
// two-kernel form gives the same bits as the fused one.
enum { ATTR_FUSED = 0, ATTR_GRAD = 1, ATTR_UPDATE = 2 };

// The variants with more loads in flight (TSNE_ATTR_PIPE=1 and 2) hold up to 48 registers per
// thread: five CTAs per SM; form 3 up to 40: six CTAs per SM.
constexpr int ATTR_PIPE_MINB = 5;
constexpr int ATTR_PIPE_GRID = 148 * ATTR_PIPE_MINB;
constexpr int ATTR_PIPE3_MINB = 6;
constexpr int ATTR_PIPE3_GRID = 148 * ATTR_PIPE3_MINB;

// PF (TSNE_ATTR_PIPE=1): each lane loads its next step's 4 entries of the row before the
// gathers of the current step; PF = 2 (TSNE_ATTR_PIPE=3): only the next step's 4 columns
// (the values, which the gathers do not wait for, are loaded with the current step). The same
// sums in the same order either way.
template <int D, int MODE, bool CONTIG, int PF>
__device__ __forceinline__ void
attr_update_rows(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
                 const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
                 Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
                 float exag4, float mom, float lr, double *__restrict__ partials, Vec<D> *__restrict__ attr)
{
    const int lane = threadIdx.x & 31, hl = lane & 15;
    const int half = (blockIdx.x * ROW_BLOCK + threadIdx.x) >> 4;
    const int nhalf = (gridDim.x * ROW_BLOCK) >> 4;
    const int use_rep = (MODE != ATTR_GRAD && rep != nullptr) ? *rep_flag : 0;
    double acc[D];
    for (int k = 0; k < D; k++) acc[k] = 0.0;
    // contig: the CTA takes the contiguous rows [r0, r1) holding its equal share of P's entries
    // (first rows whose pointers reach c E / G and (c + 1) E / G), its half-warps interleaved
    // over them, so that one SM's gathers come from one neighbourhood of the tree order
    __shared__ int s_rng[2];
    int r0 = 0, r1 = n, rounds;
    if constexpr (CONTIG) {
        if (threadIdx.x < 2) {
            const int c = blockIdx.x + threadIdx.x;
            int lo = 0;
            if (c >= (int)gridDim.x) lo = n;
            else {
                const long long target = (long long)c * rp[n] / gridDim.x;
                int hi = n;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (rp[mid] < target) lo = mid + 1;
                    else hi = mid;
                }
            }
            s_rng[threadIdx.x] = lo;
        }
        __syncthreads();
        r0 = s_rng[0];
        r1 = s_rng[1];
        rounds = (r1 - r0 + (ROW_BLOCK >> 4) - 1) / (ROW_BLOCK >> 4);
    } else {
        // both halves of a warp run the same number of rounds, so full-warp shuffles stay legal
        rounds = (n + nhalf - 1) / nhalf;
    }
    for (int rd = 0; rd < rounds; rd++) {
        const int i = CONTIG ? r0 + rd * (ROW_BLOCK >> 4) + ((int)threadIdx.x >> 4) : half + rd * nhalf;
        const bool live = i < r1;
        Vec<D> yi = vzero<D>(), opnd = vzero<D>();
        int b = 0, e = 0;
        if (live) {
            yi = Y[i];
            b = rp[i];
            e = rp[i + 1];
            if (MODE != ATTR_GRAD) {
                if (hl == 1) opnd = uY[i];
                else if (hl == 2) opnd = gains[i];
                else if (hl == 3 && use_rep) opnd = rep[i];
            }
        }
        float a[D];
#pragma unroll
        for (int k = 0; k < D; k++) a[k] = 0.f;
        if (MODE == ATTR_UPDATE) {
            if (live && hl == 0) {
                const Vec<D> s = attr[i];
#pragma unroll
                for (int k = 0; k < D; k++) a[k] = vget(s, k);
            }
        } else if (PF == 2) {
            int base = b + 4 * hl;
            int4 c4 = make_int4(0, 0, 0, 0);
            if (base < e) c4 = ld_stream_i4(col + base);
            while (base < e) {
                const int nb = base + 64;
                const float4 p4 = ld_stream_f4(val + base);
                int4 cn = c4;
                if (nb < e) cn = ld_stream_i4(col + nb);
                attr_acc<D>(yi, Y, c4.x, p4.x, a);
                attr_acc<D>(yi, Y, c4.y, p4.y, a);
                attr_acc<D>(yi, Y, c4.z, p4.z, a);
                attr_acc<D>(yi, Y, c4.w, p4.w, a);
                c4 = cn;
                base = nb;
            }
#pragma unroll
            for (int k = 0; k < D; k++)
                for (int o = 8; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        } else if (PF == 1) {
            int base = b + 4 * hl;
            int4 c4 = make_int4(0, 0, 0, 0);
            float4 p4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (base < e) { c4 = ld_stream_i4(col + base); p4 = ld_stream_f4(val + base); }
            while (base < e) {
                const int nb = base + 64;
                int4 cn = c4;
                float4 pn = p4;
                if (nb < e) { cn = ld_stream_i4(col + nb); pn = ld_stream_f4(val + nb); }
                attr_acc<D>(yi, Y, c4.x, p4.x, a);
                attr_acc<D>(yi, Y, c4.y, p4.y, a);
                attr_acc<D>(yi, Y, c4.z, p4.z, a);
                attr_acc<D>(yi, Y, c4.w, p4.w, a);
                c4 = cn;
                p4 = pn;
                base = nb;
            }
#pragma unroll
            for (int k = 0; k < D; k++)
                for (int o = 8; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        } else {
            for (int base = b + 4 * hl; base < e; base += 64) {
                const int4 c4 = ld_stream_i4(col + base);
                const float4 p4 = ld_stream_f4(val + base);
                attr_acc<D>(yi, Y, c4.x, p4.x, a);
                attr_acc<D>(yi, Y, c4.y, p4.y, a);
                attr_acc<D>(yi, Y, c4.z, p4.z, a);
                attr_acc<D>(yi, Y, c4.w, p4.w, a);
            }
#pragma unroll
            for (int k = 0; k < D; k++)
                for (int o = 8; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        }
        if (MODE == ATTR_GRAD) {
            if (live && hl == 0) {
                Vec<D> s = vzero<D>();
#pragma unroll
                for (int k = 0; k < D; k++) vset(s, k, a[k]);
                attr[i] = s;
            }
            continue;
        }
        const int src = lane & 16;
        Vec<D> u = vzero<D>(), g = vzero<D>(), r = vzero<D>();
#pragma unroll
        for (int k = 0; k < D; k++) {
            vset(u, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 1));
            vset(g, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 2));
            vset(r, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 3));
        }
        if (live && hl == 0) {
            Vec<D> yn = yi;
#pragma unroll
            for (int k = 0; k < D; k++) {
                const float gk = exag4 * a[k] - vget(r, k);
                const float uk = vget(u, k);
                float gain = (uk * gk < 0.f) ? vget(g, k) + 0.2f : vget(g, k) * 0.8f;
                gain = fmaxf(gain, 0.01f);
                const float un = mom * uk - lr * (gk * gain);
                vset(g, k, gain);
                vset(u, k, un);
                vset(yn, k, vget(yi, k) + un);
                acc[k] += (double)vget(yn, k);
            }
            uY[i] = u;
            gains[i] = g;
            Yn[i] = yn;
        }
    }
    if (MODE == ATTR_GRAD) return;
    // lanes 0 and 16 of each warp hold partial sums: fold lane 16 into lane 0
    for (int k = 0; k < D; k++) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 16);
    block_sum_warps<D>(acc, partials + (size_t)blockIdx.x * D);
}

template <int D, int MODE, bool CONTIG = false>
__global__ void __launch_bounds__(ROW_BLOCK)
k_attr_update(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
              const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
              Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
              float exag4, float mom, float lr, double *__restrict__ partials, Vec<D> *__restrict__ attr)
{
    attr_update_rows<D, MODE, CONTIG, 0>(n, rp, col, val, Y, Yn, uY, gains, rep, rep_flag, exag4, mom, lr,
                                         partials, attr);
}
template <int D, int MODE, bool CONTIG, int PF>
__global__ void __launch_bounds__(ROW_BLOCK, PF == 1 ? ATTR_PIPE_MINB : ATTR_PIPE3_MINB)
k_attr_update_pf(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
                 const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
                 Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
                 float exag4, float mom, float lr, double *__restrict__ partials, Vec<D> *__restrict__ attr)
{
    attr_update_rows<D, MODE, CONTIG, PF>(n, rp, col, val, Y, Yn, uY, gains, rep, rep_flag, exag4, mom, lr,
                                          partials, attr);
}

// The update of a rebuild iteration from its stored attractive sums, for the forms with more
// loads in flight (TSNE_ATTR_PIPE 1-3): a thread per row, rows strided over the form's grid (so
// the centring reads as many partials as after a fused step), each row's arithmetic that of
// the fused step. The half-warp-per-row update of form 0 keeps 16 lanes per row for three
// loads; this one reads and writes every array coalesced.
template <int D>
__global__ void __launch_bounds__(ROW_BLOCK)
k_update_rows(int n, const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
              Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
              const Vec<D> *__restrict__ attr, float exag4, float mom, float lr, double *__restrict__ partials)
{
    const int use_rep = rep != nullptr ? *rep_flag : 0;
    double acc[D];
#pragma unroll
    for (int k = 0; k < D; k++) acc[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> yi = Y[i], sa = attr[i];
        Vec<D> u = uY[i], g = gains[i];
        const Vec<D> r = use_rep ? rep[i] : vzero<D>();
        Vec<D> yn = yi;
#pragma unroll
        for (int k = 0; k < D; k++) {
            const float gk = exag4 * vget(sa, k) - vget(r, k);
            const float uk = vget(u, k);
            float gain = (uk * gk < 0.f) ? vget(g, k) + 0.2f : vget(g, k) * 0.8f;
            gain = fmaxf(gain, 0.01f);
            const float un = mom * uk - lr * (gk * gain);
            vset(g, k, gain);
            vset(u, k, un);
            vset(yn, k, vget(yi, k) + un);
            acc[k] += (double)vget(yn, k);
        }
        uY[i] = u;
        gains[i] = g;
        Yn[i] = yn;
    }
#pragma unroll
    for (int k = 0; k < D; k++)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
    block_sum_warps<D>(acc, partials + (size_t)blockIdx.x * D);
}

// The step as one stream of 64-entry steps per half-warp (TSNE_ATTR_PIPE=4): the next step's
// columns are loaded before the current gathers across row boundaries too: during a row's last
// step the lanes load the first columns of the half-warp's next row, whose row pointers and Y
// are loaded when the current row starts. So a row of more than one step waits on no
// row-pointer or column load, only on its gathers. Each row's sums run over the same
// lanes in the same order as in k_attr_update (same bits per row); a rebuild iteration's
// update is k_update_rows.
template <int D, int MODE, bool CONTIG>
__global__ void __launch_bounds__(ROW_BLOCK, ATTR_PIPE_MINB)
k_attr_stream(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
              const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
              Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
              float exag4, float mom, float lr, double *__restrict__ partials, Vec<D> *__restrict__ attr)
{
    static_assert(MODE != ATTR_UPDATE, "the update of a rebuild iteration is k_update_rows");
    constexpr int NHC = ROW_BLOCK >> 4;   // half-warps per CTA
    const int lane = threadIdx.x & 31, hl = lane & 15, hw = (int)threadIdx.x >> 4;
    const int half = blockIdx.x * NHC + hw;
    const int nhalf = gridDim.x * NHC;
    const int use_rep = (MODE != ATTR_GRAD && rep != nullptr) ? *rep_flag : 0;
    double acc[D];
    for (int k = 0; k < D; k++) acc[k] = 0.0;
    __shared__ int s_rng[2];
    int r0 = 0, r1 = n, rounds, first, stride;
    if constexpr (CONTIG) {
        if (threadIdx.x < 2) {
            const int c = blockIdx.x + threadIdx.x;
            int lo = 0;
            if (c >= (int)gridDim.x) lo = n;
            else {
                const long long target = (long long)c * rp[n] / gridDim.x;
                int hi = n;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (rp[mid] < target) lo = mid + 1;
                    else hi = mid;
                }
            }
            s_rng[threadIdx.x] = lo;
        }
        __syncthreads();
        r0 = s_rng[0];
        r1 = s_rng[1];
        rounds = (r1 - r0 + NHC - 1) / NHC;
        first = r0 + hw;
        stride = NHC;
    } else {
        rounds = (n + nhalf - 1) / nhalf;
        first = half;
        stride = nhalf;
    }
    // the current row (i) and the next (i + stride)
    int i = first;
    bool live = i < r1;
    Vec<D> yi = vzero<D>();
    int b = 0, e = 0;
    if (live) { yi = Y[i]; b = rp[i]; e = rp[i + 1]; }
    int4 c4 = make_int4(0, 0, 0, 0);
    if (b + 4 * hl < e) c4 = ld_stream_i4(col + b + 4 * hl);
    for (int rd = 0; rd < rounds; rd++) {
        const int i_n = i + stride;
        const bool live_n = i_n < r1;
        Vec<D> yi_n = vzero<D>(), opnd = vzero<D>();
        int nb = 0, ne = 0;
        if (live_n) { yi_n = Y[i_n]; nb = rp[i_n]; ne = rp[i_n + 1]; }
        if (MODE != ATTR_GRAD && live) {
            if (hl == 1) opnd = uY[i];
            else if (hl == 2) opnd = gains[i];
            else if (hl == 3 && use_rep) opnd = rep[i];
        }
        float a[D];
#pragma unroll
        for (int k = 0; k < D; k++) a[k] = 0.f;
        const int nch = (e - b + 63) >> 6;   // steps of this row, the same for the half-warp
        int base = b + 4 * hl;
        for (int s = 0; s < nch; s++) {
            float4 p4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (base < e) p4 = ld_stream_f4(val + base);
            const bool last = s + 1 == nch;
            const int na = last ? nb + 4 * hl : base + 64, nae = last ? ne : e;
            int4 cn = make_int4(0, 0, 0, 0);
            if (na < nae) cn = ld_stream_i4(col + na);
            if (base < e) {
                attr_acc<D>(yi, Y, c4.x, p4.x, a);
                attr_acc<D>(yi, Y, c4.y, p4.y, a);
                attr_acc<D>(yi, Y, c4.z, p4.z, a);
                attr_acc<D>(yi, Y, c4.w, p4.w, a);
            }
            c4 = cn;
            base += 64;
        }
        if (nch == 0) {   // an empty (or absent) row: the next row's first columns now
            c4 = make_int4(0, 0, 0, 0);
            if (nb + 4 * hl < ne) c4 = ld_stream_i4(col + nb + 4 * hl);
        }
#pragma unroll
        for (int k = 0; k < D; k++)
            for (int o = 8; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        if (MODE == ATTR_GRAD) {
            if (live && hl == 0) {
                Vec<D> v = vzero<D>();
#pragma unroll
                for (int k = 0; k < D; k++) vset(v, k, a[k]);
                attr[i] = v;
            }
        } else {
            const int src = lane & 16;
            Vec<D> u = vzero<D>(), g = vzero<D>(), r = vzero<D>();
#pragma unroll
            for (int k = 0; k < D; k++) {
                vset(u, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 1));
                vset(g, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 2));
                vset(r, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 3));
            }
            if (live && hl == 0) {
                Vec<D> yn = yi;
#pragma unroll
                for (int k = 0; k < D; k++) {
                    const float gk = exag4 * a[k] - vget(r, k);
                    const float uk = vget(u, k);
                    float gain = (uk * gk < 0.f) ? vget(g, k) + 0.2f : vget(g, k) * 0.8f;
                    gain = fmaxf(gain, 0.01f);
                    const float un = mom * uk - lr * (gk * gain);
                    vset(g, k, gain);
                    vset(u, k, un);
                    vset(yn, k, vget(yi, k) + un);
                    acc[k] += (double)vget(yn, k);
                }
                uY[i] = u;
                gains[i] = g;
                Yn[i] = yn;
            }
        }
        i = i_n;
        live = live_n;
        yi = yi_n;
        b = nb;
        e = ne;
    }
    if (MODE == ATTR_GRAD) return;
    for (int k = 0; k < D; k++) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 16);
    block_sum_warps<D>(acc, partials + (size_t)blockIdx.x * D);
}

// The same step with two rows per half-warp in flight (TSNE_ATTR_PIPE=2): in round rd a
// half-warp takes rows i0 and i1 = i0 + (half-warps of the split) and loads both rows' next
// 4 entries per lane before the gathers of either, so every warp keeps four streams of P
// loads and Y gathers in flight instead of two. Each row's sums run over the same lanes in
// the same order as in k_attr_update (same bits per row); lane 0 of the half-warp updates i0,
// lane 1 updates i1 (its operands come from lanes 4-6).
template <int D, int MODE, bool CONTIG>
__global__ void __launch_bounds__(ROW_BLOCK, ATTR_PIPE_MINB)
k_attr_pair(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
            const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
            Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
            float exag4, float mom, float lr, double *__restrict__ partials, Vec<D> *__restrict__ attr)
{
    constexpr int NHC = ROW_BLOCK >> 4;   // half-warps per CTA
    const int lane = threadIdx.x & 31, hl = lane & 15, hw = (int)threadIdx.x >> 4;
    const int half = blockIdx.x * NHC + hw;
    const int nhalf = gridDim.x * NHC;
    const int use_rep = (MODE != ATTR_GRAD && rep != nullptr) ? *rep_flag : 0;
    double acc[D];
    for (int k = 0; k < D; k++) acc[k] = 0.0;
    __shared__ int s_rng[2];
    int r0 = 0, r1 = n, rounds;
    if constexpr (CONTIG) {
        if (threadIdx.x < 2) {
            const int c = blockIdx.x + threadIdx.x;
            int lo = 0;
            if (c >= (int)gridDim.x) lo = n;
            else {
                const long long target = (long long)c * rp[n] / gridDim.x;
                int hi = n;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (rp[mid] < target) lo = mid + 1;
                    else hi = mid;
                }
            }
            s_rng[threadIdx.x] = lo;
        }
        __syncthreads();
        r0 = s_rng[0];
        r1 = s_rng[1];
        rounds = (r1 - r0 + 2 * NHC - 1) / (2 * NHC);
    } else {
        rounds = (n + 2 * nhalf - 1) / (2 * nhalf);
    }
    for (int rd = 0; rd < rounds; rd++) {
        const int i0 = CONTIG ? r0 + rd * 2 * NHC + hw : half + rd * 2 * nhalf;
        const int i1 = i0 + (CONTIG ? NHC : nhalf);
        const bool live0 = i0 < r1, live1 = i1 < r1;
        Vec<D> yi0 = vzero<D>(), yi1 = vzero<D>(), opnd = vzero<D>();
        int b0 = 0, e0 = 0, b1 = 0, e1 = 0;
        if (live0) {
            yi0 = Y[i0];
            b0 = rp[i0];
            e0 = rp[i0 + 1];
            if (MODE != ATTR_GRAD) {
                if (hl == 1) opnd = uY[i0];
                else if (hl == 2) opnd = gains[i0];
                else if (hl == 3 && use_rep) opnd = rep[i0];
            }
        }
        if (live1) {
            yi1 = Y[i1];
            b1 = rp[i1];
            e1 = rp[i1 + 1];
            if (MODE != ATTR_GRAD) {
                if (hl == 4) opnd = uY[i1];
                else if (hl == 5) opnd = gains[i1];
                else if (hl == 6 && use_rep) opnd = rep[i1];
            }
        }
        float a0[D], a1[D];
#pragma unroll
        for (int k = 0; k < D; k++) { a0[k] = 0.f; a1[k] = 0.f; }
        if (MODE == ATTR_UPDATE) {
            if (live0 && hl == 0) {
                const Vec<D> v = attr[i0];
#pragma unroll
                for (int k = 0; k < D; k++) a0[k] = vget(v, k);
            }
            if (live1 && hl == 1) {
                const Vec<D> v = attr[i1];
#pragma unroll
                for (int k = 0; k < D; k++) a1[k] = vget(v, k);
            }
        } else {
            for (int s0 = b0 + 4 * hl, s1 = b1 + 4 * hl; s0 < e0 || s1 < e1; s0 += 64, s1 += 64) {
                const bool g0 = s0 < e0, g1 = s1 < e1;
                int4 c0 = make_int4(0, 0, 0, 0), c1 = make_int4(0, 0, 0, 0);
                float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = make_float4(0.f, 0.f, 0.f, 0.f);
                if (g0) { c0 = ld_stream_i4(col + s0); p0 = ld_stream_f4(val + s0); }
                if (g1) { c1 = ld_stream_i4(col + s1); p1 = ld_stream_f4(val + s1); }
                if (g0) {
                    attr_acc<D>(yi0, Y, c0.x, p0.x, a0);
                    attr_acc<D>(yi0, Y, c0.y, p0.y, a0);
                    attr_acc<D>(yi0, Y, c0.z, p0.z, a0);
                    attr_acc<D>(yi0, Y, c0.w, p0.w, a0);
                }
                if (g1) {
                    attr_acc<D>(yi1, Y, c1.x, p1.x, a1);
                    attr_acc<D>(yi1, Y, c1.y, p1.y, a1);
                    attr_acc<D>(yi1, Y, c1.z, p1.z, a1);
                    attr_acc<D>(yi1, Y, c1.w, p1.w, a1);
                }
            }
#pragma unroll
            for (int k = 0; k < D; k++)
                for (int o = 8; o > 0; o >>= 1) {
                    a0[k] += __shfl_xor_sync(0xffffffffu, a0[k], o);
                    a1[k] += __shfl_xor_sync(0xffffffffu, a1[k], o);
                }
        }
        if (MODE == ATTR_GRAD) {
            Vec<D> v = vzero<D>();
            if (live0 && hl == 0) {
#pragma unroll
                for (int k = 0; k < D; k++) vset(v, k, a0[k]);
                attr[i0] = v;
            }
            if (live1 && hl == 1) {
#pragma unroll
                for (int k = 0; k < D; k++) vset(v, k, a1[k]);
                attr[i1] = v;
            }
            continue;
        }
        // lane 0 of the half updates i0 (operands from lanes 1-3), lane 1 updates i1 (lanes 4-6)
        const int src = (lane & 16) + (hl == 1 ? 3 : 0);
        const bool mine = (hl == 0 && live0) || (hl == 1 && live1);
        Vec<D> u = vzero<D>(), g = vzero<D>(), r = vzero<D>();
#pragma unroll
        for (int k = 0; k < D; k++) {
            vset(u, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 1));
            vset(g, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 2));
            vset(r, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 3));
        }
        if (mine) {
            const int i = hl == 0 ? i0 : i1;
            const Vec<D> yi = hl == 0 ? yi0 : yi1;
            Vec<D> yn = yi;
#pragma unroll
            for (int k = 0; k < D; k++) {
                const float gk = exag4 * (hl == 0 ? a0[k] : a1[k]) - vget(r, k);
                const float uk = vget(u, k);
                float gain = (uk * gk < 0.f) ? vget(g, k) + 0.2f : vget(g, k) * 0.8f;
                gain = fmaxf(gain, 0.01f);
                const float un = mom * uk - lr * (gk * gain);
                vset(g, k, gain);
                vset(u, k, un);
                vset(yn, k, vget(yi, k) + un);
                acc[k] += (double)vget(yn, k);
            }
            uY[i] = u;
            gains[i] = g;
            Yn[i] = yn;
        }
    }
    if (MODE == ATTR_GRAD) return;
    // lanes 0, 1, 16 and 17 of each warp hold partial sums: fold them into lane 0
    for (int k = 0; k < D; k++) {
        acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 16);
        acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 1);
    }
    block_sum_warps<D>(acc, partials + (size_t)blockIdx.x * D);
}

// The same step with the Y gathers served from shared memory (TSNE_ATTR_WINDOW=1 or 2; off by
// default). One CTA per SM (form 2: two) owns a contiguous range of rows holding an equal
// share of P's entries and stages the window of Y centred on it (WINP points: 128 KB, form 2
// 64 KB) once; a column
// inside the window is read from shared memory, one outside it through L1/L2. After the
// renumbering in tree order about three quarters of a point's neighbours lie inside a
// 16K-point window around it (200K-point 2D embedding of the benchmark mixture), so most
// gathers skip the L1 tag stage that bounds k_attr_update. Measured at 1M points, 2D: 0.651 ms
// per launch against k_attr_update's 0.636 ms, so not faster (it keeps 32 warps per SM
// resident instead of 64, and about a quarter of the gathers still go to L1/L2), hence off by
// default. Splitting rows by equal counts instead of equal entries made it 1.25 ms: row
// lengths follow the tree order's clusters. Used while the average CTA's row range fits in
// half a window (n <= 148 * win_pts / 2). The row of each half-warp and the summation order
// are fixed, so results are bit-reproducible, and the three modes give the same bits as one
// another.
constexpr int WIN_THREADS = 1024;
constexpr int WIN_GRID = 148;
template <int D> constexpr int win_pts() { return D == 2 ? 16384 : 8192; }

// first row i in [0, n] with rp[i] >= x (rp non-decreasing, rp[0] = 0)
__device__ __forceinline__ int first_row_at(const int *__restrict__ rp, int n, long long x)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((long long)rp[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <int D, int MODE, int WINP, int MINB>
__global__ void __launch_bounds__(WIN_THREADS, MINB)
k_attr_window(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
              const Vec<D> *__restrict__ Y, Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ uY,
              Vec<D> *__restrict__ gains, const Vec<D> *__restrict__ rep, const int *__restrict__ rep_flag,
              float exag4, float mom, float lr, double *__restrict__ partials, Vec<D> *__restrict__ attr)
{
    constexpr int WIN = WINP;
    constexpr int NH = WIN_THREADS / 16;   // half-warps per CTA
    extern __shared__ __align__(16) unsigned char win_raw[];
    Vec<D> *win = reinterpret_cast<Vec<D> *>(win_raw);
    const int lane = threadIdx.x & 31, hl = lane & 15, hw = threadIdx.x >> 4;
    // CTA b takes the rows whose entries start in [b nnz / G, (b + 1) nnz / G): equal shares of
    // P, since row lengths follow the clusters of the tree order and equal row counts would not
    // balance; the last CTA also takes the empty rows at the end
    const long long nnz = rp[n];
    const int rb = first_row_at(rp, n, (long long)blockIdx.x * nnz / gridDim.x);
    const int re = blockIdx.x + 1 == gridDim.x ? n : first_row_at(rp, n, (long long)(blockIdx.x + 1) * nnz / gridDim.x);
    int w0 = rb + (re - rb) / 2 - WIN / 2;
    w0 = max(0, min(w0, n - WIN));
    const int wl = min(WIN, n - w0);
    if (MODE != ATTR_UPDATE) {
        for (int k = threadIdx.x; k < wl; k += WIN_THREADS) win[k] = Y[w0 + k];
        __syncthreads();
    }
    const int use_rep = (MODE != ATTR_GRAD && rep != nullptr) ? *rep_flag : 0;
    double acc[D];
    for (int k = 0; k < D; k++) acc[k] = 0.0;
    // every half-warp of the CTA runs the same number of rounds (full-warp shuffles)
    const int rounds = (re - rb + NH - 1) / NH;
    for (int rd = 0; rd < rounds; rd++) {
        const int i = rb + rd * NH + hw;
        const bool live = i < re;
        Vec<D> yi = vzero<D>(), opnd = vzero<D>();
        int b = 0, e = 0;
        if (live) {
            yi = Y[i];
            b = rp[i];
            e = rp[i + 1];
            if (MODE != ATTR_GRAD) {
                if (hl == 1) opnd = uY[i];
                else if (hl == 2) opnd = gains[i];
                else if (hl == 3 && use_rep) opnd = rep[i];
            }
        }
        float a[D];
#pragma unroll
        for (int k = 0; k < D; k++) a[k] = 0.f;
        if (MODE == ATTR_UPDATE) {
            if (live && hl == 0) {
                const Vec<D> s = attr[i];
#pragma unroll
                for (int k = 0; k < D; k++) a[k] = vget(s, k);
            }
        } else {
            for (int base = b + 4 * hl; base < e; base += 64) {
                const int4 c4 = ld_stream_i4(col + base);
                const float4 p4 = ld_stream_f4(val + base);
                const int cs[4] = {c4.x, c4.y, c4.z, c4.w};
                const float ps[4] = {p4.x, p4.y, p4.z, p4.w};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const unsigned int off = (unsigned int)(cs[q] - w0);
                    const Vec<D> yj = off < (unsigned int)wl ? win[off] : __ldg(Y + cs[q]);
                    float df[D], r2 = 0.f;
#pragma unroll
                    for (int k = 0; k < D; k++) { df[k] = vget(yi, k) - vget(yj, k); r2 = fmaf(df[k], df[k], r2); }
                    const float w = ps[q] * fast_rcp(1.0f + r2);
#pragma unroll
                    for (int k = 0; k < D; k++) a[k] = fmaf(w, df[k], a[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < D; k++)
                for (int o = 8; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
        }
        if (MODE == ATTR_GRAD) {
            if (live && hl == 0) {
                Vec<D> s = vzero<D>();
#pragma unroll
                for (int k = 0; k < D; k++) vset(s, k, a[k]);
                attr[i] = s;
            }
            continue;
        }
        const int src = lane & 16;
        Vec<D> u = vzero<D>(), g = vzero<D>(), r = vzero<D>();
#pragma unroll
        for (int k = 0; k < D; k++) {
            vset(u, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 1));
            vset(g, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 2));
            vset(r, k, __shfl_sync(0xffffffffu, vget(opnd, k), src + 3));
        }
        if (live && hl == 0) {
            Vec<D> yn = yi;
#pragma unroll
            for (int k = 0; k < D; k++) {
                const float gk = exag4 * a[k] - vget(r, k);
                const float uk = vget(u, k);
                float gain = (uk * gk < 0.f) ? vget(g, k) + 0.2f : vget(g, k) * 0.8f;
                gain = fmaxf(gain, 0.01f);
                const float un = mom * uk - lr * (gk * gain);
                vset(g, k, gain);
                vset(u, k, un);
                vset(yn, k, vget(yi, k) + un);
                acc[k] += (double)vget(yn, k);
            }
            uY[i] = u;
            gains[i] = g;
            Yn[i] = yn;
        }
    }
    if (MODE == ATTR_GRAD) return;
    for (int k = 0; k < D; k++) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 16);
    block_sum_warps<D, WIN_THREADS / 32>(acc, partials + (size_t)blockIdx.x * D);
}

// Centring (reference tsne_h2pack.c:1978-1984): Y = Ynext - mean(Ynext), the mean summed
// in FP64 from the update's fixed per-block partials, identically in every block.
template <int D>
__global__ void __launch_bounds__(RED_BLOCK)
k_center(int n, const Vec<D> *__restrict__ Yn, Vec<D> *__restrict__ Y, const double *__restrict__ partials,
         int nblk, DevScalars *sc)
{
    __shared__ double mean[D];
    reduce_partials<D>(partials, nblk, mean);
    if (threadIdx.x == 0) {
        for (int k = 0; k < D; k++) mean[k] /= (double)n;
        if (blockIdx.x == 0)
            for (int k = 0; k < D; k++) sc->mean[k] = mean[k];
    }
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Vec<D> v = Yn[i];
#pragma unroll
        for (int k = 0; k < D; k++) vset(v, k, (float)((double)vget(v, k) - mean[k]));
        Y[i] = v;
    }
}

// Exact off-diagonal sums s_i = sum_{j != i} K_ij, v_i = sum_{j != i} K_ij y_j
// (reference tsne_h2pack.c:404-491): one thread per target, sources staged through
// shared memory 256 at a time, FP32 per tile and FP64 across tiles.
template <int D>
__global__ void __launch_bounds__(256)
k_exact_sv(int n, const Vec<D> *__restrict__ Y, float *__restrict__ s, Vec<D> *__restrict__ v)
{
    __shared__ Vec<D> sh[256];
    const int i = blockIdx.x * 256 + threadIdx.x;
    const Vec<D> yi = (i < n) ? Y[i] : vzero<D>();
    double S = 0.0, V[D];
    for (int k = 0; k < D; k++) V[k] = 0.0;
    for (int base = 0; base < n; base += 256) {
        __syncthreads();
        if (base + (int)threadIdx.x < n) sh[threadIdx.x] = Y[base + threadIdx.x];
        __syncthreads();
        const int cnt = min(256, n - base);
        float ts = 0.f, tv[D];
#pragma unroll
        for (int k = 0; k < D; k++) tv[k] = 0.f;
        for (int j = 0; j < cnt; j++) {
            const Vec<D> yj = sh[j];
            float w = rkernel(dist2(yi, yj));
            w = (base + j == i) ? 0.f : w;
            ts += w;
#pragma unroll
            for (int k = 0; k < D; k++) tv[k] = fmaf(w, vget(yj, k), tv[k]);
        }
        S += ts;
        for (int k = 0; k < D; k++) V[k] += tv[k];
    }
    if (i < n) {
        s[i] = (float)S;
        Vec<D> o = vzero<D>();
        for (int k = 0; k < D; k++) vset(o, k, (float)V[k]);
        v[i] = o;
    }
}

// Z identity (reference tsne_h2pack.c:558-590): Z = sum s + 2 sum |y|^2 s - 2 sum y.v,
// three FP64 sums over fixed blocks.
template <int D>
__global__ void __launch_bounds__(RED_BLOCK)
k_z_part(int n, const Vec<D> *__restrict__ Yp, const float *__restrict__ s, const Vec<D> *__restrict__ v,
         double *__restrict__ partials)
{
    double t[3] = {0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> y = Yp[i], vv = v[i];
        double yy = 0.0, yv = 0.0;
#pragma unroll
        for (int k = 0; k < D; k++) {
            const double yk = vget(y, k);
            yy += yk * yk;
            yv += yk * (double)vget(vv, k);
        }
        t[0] += s[i];
        t[1] += yy * s[i];
        t[2] += yv;
    }
    __shared__ double sh[RED_BLOCK][3];
    for (int k = 0; k < 3; k++) sh[threadIdx.x][k] = t[k];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int k = 0; k < 3; k++) sh[threadIdx.x][k] += sh[threadIdx.x + st][k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; k++) partials[(size_t)blockIdx.x * 3 + k] = sh[0][k];
}

// Force assembly (reference tsne_h2pack.c:604-627): F_i = (4/Z)(y_i s_i - v_i), written in
// point order (perm maps tree positions to points). On the H2 path a non-positive or
// non-finite Z skips the force, as the reference does.
template <int D>
__global__ void __launch_bounds__(RED_BLOCK)
k_force(int n, const Vec<D> *__restrict__ Yp, const float *__restrict__ s, const Vec<D> *__restrict__ v,
        const int *__restrict__ perm, Vec<D> *__restrict__ F, DevScalars *sc,
        const double *__restrict__ partials, int nblk, int h2_path, int keep_rep)
{
    __shared__ double tz[3];
    reduce_partials<3>(partials, nblk, tz);
    const double Z = tz[0] + 2.0 * tz[1] - 2.0 * tz[2];
    const bool ok = !h2_path || (Z > 0.0 && isfinite(Z));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->Z = ok ? Z : 1.0;
        sc->force_ok = ok ? 1 : 0;
        sc->bad_z = ok ? 0 : 1;
        if (ok && keep_rep) { sc->rep_valid = 1; sc->rep_Z = Z; }
    }
    if (!ok) return;
    const double c = 4.0 / Z;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> y = Yp[i], vv = v[i];
        const double si = s[i];
        Vec<D> f = vzero<D>();
#pragma unroll
        for (int k = 0; k < D; k++) vset(f, k, (float)(c * ((double)vget(y, k) * si - (double)vget(vv, k))));
        F[perm ? perm[i] : i] = f;
    }
}

// KL(P || Q) of the exaggerated P with q_ij = 1 / ((1 + |y_i - y_j|^2) Z)
// (reference tsne_h2pack.c:1870-1895), FP64 per entry.
template <int D>
__global__ void __launch_bounds__(ROW_BLOCK)
k_kl(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
     const Vec<D> *__restrict__ Y, double exag, const DevScalars *__restrict__ sc, double *__restrict__ partials)
{
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * (ROW_BLOCK / 32) + (threadIdx.x >> 5);
    const int nwarp = gridDim.x * (ROW_BLOCK / 32);
    const double Z = sc->Z;
    double acc[1] = {0.0};
    for (int i = warp; i < n; i += nwarp) {
        const Vec<D> yi = Y[i];
        double r = 0.0;
        for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) {
            const double p = (double)val[e] * exag;
            const Vec<D> yj = Y[col[e]];
            double r2 = 0.0;
#pragma unroll
            for (int k = 0; k < D; k++) { const double df = (double)vget(yi, k) - (double)vget(yj, k); r2 += df * df; }
            const double q = 1.0 / ((1.0 + r2) * Z);
            if (p > 1e-12 && q > 1e-12) r += p * log(p / q);
        }
        r = warp_sum(r);
        if (lane == 0) acc[0] += r;
    }
    block_sum_warps<1>(acc, partials + blockIdx.x);
}

__global__ void __launch_bounds__(RED_BLOCK) k_kl_final(const double *__restrict__ partials, int nblk, DevScalars *sc)
{
    __shared__ double out[1];
    reduce_partials<1>(partials, nblk, out);
    if (threadIdx.x == 0) sc->kl = out[0];
}

// grad (SoA double, reference layout) += scale * attractive sums
template <int D>
__global__ void __launch_bounds__(ROW_BLOCK)
k_attr_only(int n, const int *__restrict__ rp, const int *__restrict__ col, const float *__restrict__ val,
            const Vec<D> *__restrict__ Y, double scale, double *__restrict__ grad)
{
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * (ROW_BLOCK / 32) + (threadIdx.x >> 5);
    const int nwarp = gridDim.x * (ROW_BLOCK / 32);
    for (int i = warp; i < n; i += nwarp) {
        float a[D];
#pragma unroll
        for (int k = 0; k < D; k++) a[k] = 0.f;
        row_attr<D>(rp[i], rp[i + 1], lane, Y[i], col, val, Y, a);
        if (lane == 0)
            for (int k = 0; k < D; k++) grad[(size_t)k * n + i] += scale * (double)a[k];
    }
}

template <int D>
__global__ void k_soa_to_vec(int n, const double *__restrict__ soa, Vec<D> *__restrict__ v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Vec<D> o = vzero<D>();
        for (int k = 0; k < D; k++) vset(o, k, (float)soa[(size_t)k * n + i]);
        v[i] = o;
    }
}

template <int D>
__global__ void k_vec_to_soa(int n, const Vec<D> *__restrict__ v, double *__restrict__ soa)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Vec<D> x = v[i];
        for (int k = 0; k < D; k++) soa[(size_t)k * n + i] = (double)vget(x, k);
    }
}

template <int D>
__global__ void k_fill_vec(int n, Vec<D> *__restrict__ v, float value)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Vec<D> o = vzero<D>();
        for (int k = 0; k < D; k++) vset(o, k, value);
        v[i] = o;
    }
}

template <int D>
__global__ void k_permute_vec(int n, const int *__restrict__ ord, const Vec<D> *__restrict__ src,
                              Vec<D> *__restrict__ dst)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[ord[i]];
}

__global__ void k_permute_int(int n, const int *__restrict__ ord, const int *__restrict__ src,
                              int *__restrict__ dst, int identity_src)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = identity_src ? ord[i] : src[ord[i]];
}

__global__ void k_invert_perm(int n, const int *__restrict__ ord, int *__restrict__ inv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) inv[ord[i]] = i;
}

__global__ void k_row_len(int n, const int *__restrict__ ord, const int *__restrict__ rp, int *__restrict__ len)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = ord[k];
        len[k] = rp[i + 1] - rp[i];
    }
}

// Renumbered rows (reference tsne_reorder.c:112-167): new row k is old row ord[k] with its
// columns mapped through inv, one warp per row, four entries per lane (rows are padded to
// multiples of 4, so every row starts on a 16-byte boundary). The entries keep their order
// inside the row.
__global__ void __launch_bounds__(ROW_BLOCK)
k_row_gather(int n, const int *__restrict__ ord, const int *__restrict__ inv, const int *__restrict__ rp_old,
             const int *__restrict__ col_old, const float *__restrict__ val_old, const int *__restrict__ rp_new,
             int *__restrict__ col_new, float *__restrict__ val_new)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarp = (gridDim.x * blockDim.x) >> 5;
    for (int k = warp; k < n; k += nwarp) {
        const int i = ord[k], b = rp_old[i], len = rp_old[i + 1] - b, o = rp_new[k];
        for (int e = 4 * lane; e < len; e += 128) {
            int4 c = ld_stream_i4(col_old + b + e);
            const float4 v = ld_stream_f4(val_old + b + e);
            c.x = inv[c.x]; c.y = inv[c.y]; c.z = inv[c.z]; c.w = inv[c.w];
            *reinterpret_cast<int4 *>(col_new + o + e) = c;
            *reinterpret_cast<float4 *>(val_new + o + e) = v;
        }
    }
}

// Conditional P_j|i by bisection on beta over min-shifted squared distances, FP64
// (reference tsne_utils.c:952-1005): one warp per row; the search state is uniform
// across the warp and every sum is a warp reduction.
__global__ void __launch_bounds__(256)
k_pcal(int n, const int *__restrict__ indptr, const double *__restrict__ dist, double perplexity,
       double *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarp = (gridDim.x * blockDim.x) >> 5;
    const double target = log(perplexity);
    for (int i = warp; i < n; i += nwarp) {
        const int b = indptr[i], k = indptr[i + 1] - b;
        if (k <= 0) continue;
        double dmin = INFINITY;
        for (int j = lane; j < k; j += 32) { const double d = dist[b + j]; dmin = fmin(dmin, d * d); }
        for (int o = 16; o > 0; o >>= 1) dmin = fmin(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
        double beta = 1.0, lo = 0.0, hi = 0.0, sp = 1.0;
        bool have_lo = false, have_hi = false;
        double beta_eval = beta;
        for (int it = 0; it < 200; it++) {
            double a = 0.0, c = 0.0;
            for (int j = lane; j < k; j += 32) {
                const double d = dist[b + j];
                const double dd = d * d - dmin;
                const double p = exp(-beta * dd);
                a += p;
                c += dd * p;
            }
            a = warp_sum(a);
            c = warp_sum(c);
            sp = a;
            beta_eval = beta;
            const double H = log(a) + beta * c / a;
            const double diff = H - target;
            if (fabs(diff) < 1e-5) break;
            if (diff > 0.0) { lo = beta; have_lo = true; beta = have_hi ? 0.5 * (beta + hi) : 2.0 * beta; }
            else            { hi = beta; have_hi = true; beta = have_lo ? 0.5 * (beta + lo) : 0.5 * beta; }
        }
        const double inv = 1.0 / sp;
        for (int j = lane; j < k; j += 32) {
            const double d = dist[b + j];
            out[b + j] = exp(-beta_eval * (d * d - dmin)) * inv;
        }
    }
}

constexpr int EW_BLOCK = 256;
inline int ew_grid(int n) { int g = ceil_div(n, EW_BLOCK); return g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g); }

}  // namespace

// ---------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------
// The shared-memory window forms of the attractive step (k_attr_window), chosen by
// TSNE_ATTR_WINDOW: 1, one CTA per SM with a 128 KB window; 2 (2D; 3D takes form 1, its
// update spills at 32 registers), two CTAs per SM with 64 KB windows (at most 32 registers
// per thread, so twice the resident warps). A form is taken
// while the average CTA's row range fits in half its window; all three modes and the
// centring follow the same rule, so a step's kernels always agree on the row split. 0 (the
// default): k_attr_update. Measured at 1M points, 2D: form 2 takes 1.40 ms per launch, form 1
// 0.651 ms, k_attr_update 0.62 ms.
template <int D>
int window_form(int n)
{
    static const int form = [] {
        const char *e = getenv("TSNE_ATTR_WINDOW");
        const int v = e != nullptr ? atoi(e) : 0;
        return (v == 1 || v == 2) ? v : 0;
    }();
    const int f = (D == 3 && form == 2) ? 1 : form;
    if (f == 0) return 0;
    return ceil_div(n, f * WIN_GRID) <= win_pts<D>() / f / 2 ? f : 0;
}
// Form of the attractive step, TSNE_ATTR_PIPE: 0 k_attr_update (32 registers in 2D, eight CTAs
// per SM); 1 the same with the next step's entries loaded ahead (48 registers, five CTAs per
// SM); 2 k_attr_pair (two rows per half-warp, five CTAs per SM); 3 the next step's columns
// loaded ahead (40 registers, six CTAs per SM); 4 k_attr_stream (the column loads ahead across
// the rows of a half-warp, five CTAs per SM). Measured at 1M points, 2D, per launch: 0.619,
// 0.608, 0.616, 0.592 and 0.634 ms, so 2D takes form 3 by default. In 3D the fused kernel holds 48
// registers in every form and form 3 spills there; form 1 measured no faster than form 0 at
// 500K points (0.352 against 0.348 ms per launch), so 3D keeps form 0. The attractive sums of a
// rebuild iteration follow the form; their update is k_update_rows for forms 1-3.
template <int D>
int attr_pipe()
{
    const char *e = getenv("TSNE_ATTR_PIPE");
    if (e == nullptr || *e == '\0') return D == 2 ? 3 : 0;
    const int x = atoi(e);
    return (x >= 1 && x <= 4) ? x : 0;
}
template <int D>
int attr_blocks(int n)
{
    const int form = window_form<D>(n);
    if (form != 0) return form * WIN_GRID;
    const int pipe = attr_pipe<D>();
    return pipe == 3 ? ATTR_PIPE3_GRID : pipe != 0 ? ATTR_PIPE_GRID : ROW_GRID;
}
template <int D, int MODE, int FORM>
void launch_window_form(cudaStream_t st, int n, const int *rp, const int *col, const float *val, const void *Y,
                        void *Ynext, void *uY, void *gains, const void *rep, const int *rep_flag, float exag4,
                        float mom, float lr, double *partials, void *attr)
{
    constexpr int WINP = win_pts<D>() / FORM;
    constexpr size_t smem = MODE == ATTR_UPDATE ? 0 : sizeof(Vec<D>) * (size_t)WINP;
    // the window's shared memory, and (two CTAs per SM) a carve-out that holds both windows
    static const cudaError_t attr_set =
        FORM == 2 ? (cudaFuncSetAttribute(k_attr_window<D, MODE, WINP, FORM>,
                                          cudaFuncAttributePreferredSharedMemoryCarveout,
                                          (int)cudaSharedmemCarveoutMaxShared),
                     cudaFuncSetAttribute(k_attr_window<D, MODE, WINP, FORM>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))
                  : cudaFuncSetAttribute(k_attr_window<D, MODE, WINP, FORM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    (void)attr_set;
    k_attr_window<D, MODE, WINP, FORM><<<FORM * WIN_GRID, WIN_THREADS, smem, st>>>(
        n, rp, col, val, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains, (const Vec<D> *)rep,
        rep_flag, exag4, mom, lr, partials, (Vec<D> *)attr);
}
template <int D, int MODE>
void launch_window(cudaStream_t st, int n, const int *rp, const int *col, const float *val, const void *Y,
                   void *Ynext, void *uY, void *gains, const void *rep, const int *rep_flag, float exag4, float mom,
                   float lr, double *partials, void *attr)
{
    if (window_form<D>(n) == 1)
        launch_window_form<D, MODE, 1>(st, n, rp, col, val, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom, lr,
                                       partials, attr);
    else
        launch_window_form<D, MODE, 2>(st, n, rp, col, val, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom, lr,
                                       partials, attr);
}

// Every CTA of the attractive step takes a contiguous range of rows (equal shares of P's
// entries) instead of rows dealt round-robin, so one SM's gathers come from one neighbourhood of
// the tree order (measured at 1M points: 0.622 ms per launch against 0.634 round-robin);
// TSNE_ATTR_CONTIG=0 restores the round-robin split. All three modes follow the same split.
int attr_contig()
{
    static const int v = [] {
        const char *e = getenv("TSNE_ATTR_CONTIG");
        return e != nullptr && atoi(e) == 0 ? 0 : 1;
    }();
    return v;
}

template <int D, int MODE, bool CONTIG>
void launch_attr_rows(cudaStream_t st, int n, const int *rp, const int *col, const float *val, const void *Y,
                      void *Ynext, void *uY, void *gains, const void *rep, const int *rep_flag, float exag4,
                      float mom, float lr, double *partials, void *attr)
{
    const int pipe = attr_pipe<D>();
    if constexpr (MODE != ATTR_UPDATE) {
        if (pipe == 4) {
            k_attr_stream<D, MODE, CONTIG><<<ATTR_PIPE_GRID, ROW_BLOCK, 0, st>>>(
                n, rp, col, val, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains,
                (const Vec<D> *)rep, rep_flag, exag4, mom, lr, partials, (Vec<D> *)attr);
            return;
        }
    }
    if (pipe == 2)
        k_attr_pair<D, MODE, CONTIG><<<ATTR_PIPE_GRID, ROW_BLOCK, 0, st>>>(
            n, rp, col, val, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains,
            (const Vec<D> *)rep, rep_flag, exag4, mom, lr, partials, (Vec<D> *)attr);
    else if (pipe == 3)
        k_attr_update_pf<D, MODE, CONTIG, 2><<<ATTR_PIPE3_GRID, ROW_BLOCK, 0, st>>>(
            n, rp, col, val, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains,
            (const Vec<D> *)rep, rep_flag, exag4, mom, lr, partials, (Vec<D> *)attr);
    else if (pipe == 1)
        k_attr_update_pf<D, MODE, CONTIG, 1><<<ATTR_PIPE_GRID, ROW_BLOCK, 0, st>>>(
            n, rp, col, val, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains,
            (const Vec<D> *)rep, rep_flag, exag4, mom, lr, partials, (Vec<D> *)attr);
    else
        k_attr_update<D, MODE, CONTIG><<<ROW_GRID, ROW_BLOCK, 0, st>>>(
            n, rp, col, val, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains,
            (const Vec<D> *)rep, rep_flag, exag4, mom, lr, partials, (Vec<D> *)attr);
}
template <int D, int MODE>
void launch_attr_any(cudaStream_t st, int n, const int *rp, const int *col, const float *val, const void *Y,
                     void *Ynext, void *uY, void *gains, const void *rep, const int *rep_flag, float exag4,
                     float mom, float lr, double *partials, void *attr)
{
    if (attr_contig())
        launch_attr_rows<D, MODE, true>(st, n, rp, col, val, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom, lr,
                                        partials, attr);
    else
        launch_attr_rows<D, MODE, false>(st, n, rp, col, val, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom, lr,
                                         partials, attr);
}

template <int D>
void launch_attr_update(cudaStream_t st, int n, const int *rp, const int *col, const float *val,
                        const void *Y, void *Ynext, void *uY, void *gains, const void *rep,
                        const int *rep_flag, float exag4, float mom, float lr, double *partials)
{
    if (window_form<D>(n) != 0) {
        launch_window<D, ATTR_FUSED>(st, n, rp, col, val, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom, lr,
                                     partials, nullptr);
        return;
    }
    launch_attr_any<D, ATTR_FUSED>(st, n, rp, col, val, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom, lr,
                                   partials, nullptr);
}
template <int D>
void launch_attr_grad(cudaStream_t st, int n, const int *rp, const int *col, const float *val, const void *Y,
                      void *attr)
{
    if (window_form<D>(n) != 0) {
        launch_window<D, ATTR_GRAD>(st, n, rp, col, val, Y, nullptr, nullptr, nullptr, nullptr, nullptr, 0.f, 0.f,
                                    0.f, nullptr, attr);
        return;
    }
    launch_attr_any<D, ATTR_GRAD>(st, n, rp, col, val, Y, nullptr, nullptr, nullptr, nullptr, nullptr, 0.f, 0.f,
                                  0.f, nullptr, attr);
}
template <int D>
void launch_update(cudaStream_t st, int n, const int *rp, const void *Y, void *Ynext, void *uY, void *gains,
                   const void *rep, const int *rep_flag, const void *attr, float exag4, float mom, float lr,
                   double *partials)
{
    if (window_form<D>(n) != 0) {
        launch_window<D, ATTR_UPDATE>(st, n, rp, nullptr, nullptr, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom,
                                      lr, partials, const_cast<void *>(attr));
        return;
    }
    if (attr_pipe<D>() != 0) {
        k_update_rows<D><<<attr_blocks<D>(n), ROW_BLOCK, 0, st>>>(
            n, (const Vec<D> *)Y, (Vec<D> *)Ynext, (Vec<D> *)uY, (Vec<D> *)gains, (const Vec<D> *)rep, rep_flag,
            (const Vec<D> *)attr, exag4, mom, lr, partials);
        return;
    }
    launch_attr_any<D, ATTR_UPDATE>(st, n, rp, nullptr, nullptr, Y, Ynext, uY, gains, rep, rep_flag, exag4, mom,
                                    lr, partials, const_cast<void *>(attr));
}

template <int D>
void launch_center(cudaStream_t st, int n, const void *Ynext, void *Ycur, const double *partials,
                   DevScalars *sc, const void *, double *)
{
    const int nblk = attr_blocks<D>(n);
    k_center<D><<<ew_grid(n), RED_BLOCK, 0, st>>>(n, (const Vec<D> *)Ynext, (Vec<D> *)Ycur, partials, nblk, sc);
}

template <int D>
void launch_exact_sv(cudaStream_t st, int n, const void *Y, float *s, void *v)
{
    k_exact_sv<D><<<ceil_div(n, 256), 256, 0, st>>>(n, (const Vec<D> *)Y, s, (Vec<D> *)v);
}

template <int D>
void launch_z_force(cudaStream_t st, int n, const void *Ypts, const float *s, const void *v,
                    const int *perm, void *rep, DevScalars *sc, double *partials, int h2_path,
                    int keep_rep)
{
    const int nblk = 148 * 2;
    k_z_part<D><<<nblk, RED_BLOCK, 0, st>>>(n, (const Vec<D> *)Ypts, s, (const Vec<D> *)v, partials);
    k_force<D><<<ew_grid(n), RED_BLOCK, 0, st>>>(n, (const Vec<D> *)Ypts, s, (const Vec<D> *)v, perm,
                                                 (Vec<D> *)rep, sc, partials, nblk, h2_path, keep_rep);
}

template <int D>
void launch_kl(cudaStream_t st, int n, const int *rp, const int *col, const float *val,
               const void *Y, double exag, DevScalars *sc, double *partials)
{
    k_kl<D><<<ROW_GRID, ROW_BLOCK, 0, st>>>(n, rp, col, val, (const Vec<D> *)Y, exag, sc, partials);
    k_kl_final<<<1, RED_BLOCK, 0, st>>>(partials, ROW_GRID, sc);
}

template <int D>
void launch_attr_only(cudaStream_t st, int n, const int *rp, const int *col, const float *val,
                      const void *Y, double scale, double *grad_soa)
{
    k_attr_only<D><<<ROW_GRID, ROW_BLOCK, 0, st>>>(n, rp, col, val, (const Vec<D> *)Y, scale, grad_soa);
}

template <int D>
void launch_soa_to_vec(cudaStream_t st, int n, const double *soa, void *vec)
{
    k_soa_to_vec<D><<<ew_grid(n), EW_BLOCK, 0, st>>>(n, soa, (Vec<D> *)vec);
}

template <int D>
void launch_vec_to_soa(cudaStream_t st, int n, const void *vec, double *soa)
{
    k_vec_to_soa<D><<<ew_grid(n), EW_BLOCK, 0, st>>>(n, (const Vec<D> *)vec, soa);
}

template <int D>
void launch_fill_vec(cudaStream_t st, int n, void *vec, float value)
{
    k_fill_vec<D><<<ew_grid(n), EW_BLOCK, 0, st>>>(n, (Vec<D> *)vec, value);
}

template <int D>
void launch_permute_vec(cudaStream_t st, int n, const int *ord, const void *src, void *dst)
{
    k_permute_vec<D><<<ew_grid(n), EW_BLOCK, 0, st>>>(n, ord, (const Vec<D> *)src, (Vec<D> *)dst);
}

void launch_permute_int(cudaStream_t st, int n, const int *ord, const int *src, int *dst, int identity_src)
{
    k_permute_int<<<ew_grid(n), EW_BLOCK, 0, st>>>(n, ord, src, dst, identity_src);
}

void launch_invert_perm(cudaStream_t st, int n, const int *ord, int *inv)
{
    k_invert_perm<<<ew_grid(n), EW_BLOCK, 0, st>>>(n, ord, inv);
}

void launch_row_len(cudaStream_t st, int n, const int *ord, const int *rp_old, int *len_new)
{
    k_row_len<<<ew_grid(n), EW_BLOCK, 0, st>>>(n, ord, rp_old, len_new);
}

void launch_row_gather(cudaStream_t st, int n, const int *ord, const int *inv, const int *rp_old,
                       const int *col_old, const float *val_old, const int *rp_new, int *col_new, float *val_new)
{
    k_row_gather<<<ROW_GRID, ROW_BLOCK, 0, st>>>(n, ord, inv, rp_old, col_old, val_old, rp_new, col_new, val_new);
}

void launch_pcal(cudaStream_t st, int n, const int *indptr, const double *dist, double perplexity,
                 double *out)
{
    k_pcal<<<ROW_GRID, 256, 0, st>>>(n, indptr, dist, perplexity, out);
}

#define TSNE_INST(D)                                                                              \
    template void launch_attr_update<D>(cudaStream_t, int, const int *, const int *, const float *,  \
                                        const void *, void *, void *, void *, const void *,          \
                                        const int *, float, float, float, double *);                 \
    template void launch_attr_grad<D>(cudaStream_t, int, const int *, const int *, const float *,    \
                                      const void *, void *);                                         \
    template void launch_update<D>(cudaStream_t, int, const int *, const void *, void *, void *,     \
                                   void *, const void *, const int *, const void *, float, float,    \
                                   float, double *);                                                 \
    template void launch_center<D>(cudaStream_t, int, const void *, void *, const double *,         \
                                   DevScalars *, const void *, double *);                            \
    template void launch_exact_sv<D>(cudaStream_t, int, const void *, float *, void *);             \
    template void launch_z_force<D>(cudaStream_t, int, const void *, const float *, const void *,   \
                                    const int *, void *, DevScalars *, double *, int, int);          \
    template void launch_kl<D>(cudaStream_t, int, const int *, const int *, const float *,          \
                               const void *, double, DevScalars *, double *);                       \
    template void launch_attr_only<D>(cudaStream_t, int, const int *, const int *, const float *,   \
                                      const void *, double, double *);                              \
    template void launch_soa_to_vec<D>(cudaStream_t, int, const double *, void *);                  \
    template void launch_vec_to_soa<D>(cudaStream_t, int, const void *, double *);                  \
    template void launch_fill_vec<D>(cudaStream_t, int, void *, float);                             \
    template void launch_permute_vec<D>(cudaStream_t, int, const int *, const void *, void *);

TSNE_INST(2)
TSNE_INST(3)

}  // namespace tsne
