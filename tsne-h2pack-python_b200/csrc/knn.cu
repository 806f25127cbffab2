// The k-NN graph on the device, and the feature-space entry points of the C ABI built on it:
// tsne_knn_graph (the exact graph the reference's Python front ends compute on the host,
// tsne_h2pack/_knn_methods.py:71-119), compute_sparse_P (reference src/tsne_utils.c:828-933,
// there a ball-tree k-NN on the host), tsne_init and tsne_fit_transform. The exact k nearest
// neighbours (k = 3 * perplexity for compute_sparse_P) come from a tiled device scan, the
// conditional P from the device beta bisection, and P is symmetrised as P + P^T and normalised
// on the device (pjoint.cu), as the reference's Python backend does on the host
// (tsne_h2pack/_backend.py:709-718).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <thread>
#include <chrono>
#include <climits>
#include <utility>
#include <vector>

#include "common.cuh"
#include "devbuf.h"
#include "kernels.h"
#include "pjoint.h"
#include "../../include/tsne_h2pack.h"

using namespace tsne;

namespace {

// ---------------------------------------------------------------------------------
// Exact k nearest neighbours by a tiled scan. A CTA of 256 threads owns 64 query rows and
// walks every point in tiles of 128, starting at its own tile and wrapping around (the
// nearest points tend to lie near the query in the input order, so the per-row threshold
// tightens early). Distances: d^2 = |q|^2 + |p|^2 - 2 q.p in FP32, the dot products
// register-tiled (each thread 4 queries x 8 points, operands staged dimension-major in shared
// memory). A distance below its row's threshold (the k-th best so far; +inf until k are known)
// is appended to the row's candidate buffer in shared memory; after a tile, rows whose buffer
// holds more than KBUF entries are merged by one warp (bitonic sort of the buffer by (d^2,
// index), keep the first k, new threshold = the k-th). Ties keep the smaller index. The output
// rows are sorted by index (as the calibration expects them); the reported distances (not
// squared) are recomputed from the coordinates' differences.
// ---------------------------------------------------------------------------------
constexpr int KNN_MAX_K = 128;          // largest k of the tiled scan (perplexity <= 42)
constexpr int KQ = 64;                  // queries per CTA
constexpr int KT = 128;                 // points per tile
constexpr int KBUF = 128;               // buffer slots that hold the current best k
constexpr int KCAP = KBUF + KT;         // a row's buffer: best k + one tile of candidates
constexpr int KNN_THREADS = 256;
constexpr int KNN_WARP_MAX_K = 256;

// One warp per query (k above the tiled scan's limit, or more than 120 dimensions): distances to every point in chunks of 32, a sorted top-k list in
// shared memory updated by warp-cooperative insertion. Ties keep the smaller index.
__global__ void __launch_bounds__(128)
k_knn_warp(int n, int dim, const float *__restrict__ X, int k, int *__restrict__ out_idx, float *__restrict__ out_d2)
{
    __shared__ float sd[4][KNN_WARP_MAX_K];
    __shared__ int si[4][KNN_WARP_MAX_K];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *bd = sd[w];
    int *bi = si[w];
    for (int q = blockIdx.x * 4 + w; q < n; q += gridDim.x * 4) {
        for (int j = lane; j < k; j += 32) { bd[j] = INFINITY; bi[j] = INT_MAX; }
        __syncwarp();
        const float *xq = X + (size_t)q * dim;
        for (int base = 0; base < n; base += 32) {
            const int j = base + lane;
            float d2 = INFINITY;
            if (j < n && j != q) {
                const float *xj = X + (size_t)j * dim;
                float acc = 0.f;
                for (int c = 0; c < dim; c++) { const float df = xq[c] - xj[c]; acc = fmaf(df, df, acc); }
                d2 = acc;
            }
            unsigned cand = __ballot_sync(0xffffffffu, d2 < bd[k - 1] || (d2 == bd[k - 1] && j < bi[k - 1]));
            while (cand) {
                const int src = __ffs(cand) - 1;
                cand &= cand - 1;
                const float cd = __shfl_sync(0xffffffffu, d2, src);
                const int cj = __shfl_sync(0xffffffffu, j, src);
                if (!(cd < bd[k - 1] || (cd == bd[k - 1] && cj < bi[k - 1]))) continue;
                // position = number of entries strictly before (cd, cj)
                int pos = 0;
                for (int t = lane; t < k; t += 32) pos += (bd[t] < cd || (bd[t] == cd && bi[t] < cj));
                pos = warp_sum(pos);
                // shift the tail right by one, from the end
                for (int t0 = k - 1; t0 > pos; t0 -= 32) {
                    const int t = t0 - lane;
                    float vd = 0.f; int vi = 0;
                    const bool act = t > pos;
                    if (act) { vd = bd[t - 1]; vi = bi[t - 1]; }
                    __syncwarp();
                    if (act) { bd[t] = vd; bi[t] = vi; }
                    __syncwarp();
                }
                if (lane == 0) { bd[pos] = cd; bi[pos] = cj; }
                __syncwarp();
            }
        }
        for (int j = lane; j < k; j += 32) { out_idx[(size_t)q * k + j] = bi[j]; out_d2[(size_t)q * k + j] = bd[j]; }
        __syncwarp();
    }
}


size_t knn_smem_bytes(int dp)
{
    return sizeof(float) * ((size_t)dp * (KQ + KT) + KQ + KT + 2 * KQ) + sizeof(int) * 2 * KQ +
           (sizeof(float) + sizeof(int)) * (size_t)KQ * KCAP;
}

// one warp sorts a row's buffer (KCAP = 256 entries, +inf / INT_MAX beyond `m`) ascending by
// (key, tie) with a bitonic network
__device__ void warp_bitonic(float *key, int *tie, int lane)
{
    for (int size = 2; size <= KCAP; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < KCAP / 2; t += 32) {
                const int a = 2 * stride * (t / stride) + (t % stride), b = a + stride;
                const bool up = (a & size) == 0;
                const float ka = key[a], kb = key[b];
                const int ia = tie[a], ib = tie[b];
                const bool gt = ka > kb || (ka == kb && ia > ib);
                if (gt == up) { key[a] = kb; key[b] = ka; tie[a] = ib; tie[b] = ia; }
            }
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(KNN_THREADS, 1)
k_knn_tiled(int n, int dp, int k, const float *__restrict__ X, const float *__restrict__ xn,
            int *__restrict__ out_idx, float *__restrict__ out_d)
{
    extern __shared__ float smem[];
    float *qs = smem;                         // [dp][KQ]
    float *ps = qs + (size_t)dp * KQ;         // [dp][KT]
    float *qn = ps + (size_t)dp * KT;         // [KQ]
    float *pn = qn + KQ;                      // [KT]
    float *tau = pn + KT;                     // [KQ] threshold: the k-th best d^2 so far
    int *taui = reinterpret_cast<int *>(tau + KQ);       // [KQ] its index (ties)
    int *cnt = taui + KQ;                     // [KQ]
    float *bd = reinterpret_cast<float *>(cnt + KQ);     // [KQ][KCAP]
    int *bi = reinterpret_cast<int *>(bd + (size_t)KQ * KCAP);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int q0 = blockIdx.x * KQ;
    const int dq = dp >> 2;
    for (int idx = tid; idx < KQ * dq; idx += KNN_THREADS) {
        const int q = idx % KQ, c4 = idx / KQ;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q0 + q < n) v = *reinterpret_cast<const float4 *>(X + (size_t)(q0 + q) * dp + 4 * c4);
        qs[(4 * c4 + 0) * KQ + q] = v.x;
        qs[(4 * c4 + 1) * KQ + q] = v.y;
        qs[(4 * c4 + 2) * KQ + q] = v.z;
        qs[(4 * c4 + 3) * KQ + q] = v.w;
    }
    if (tid < KQ) {
        qn[tid] = q0 + tid < n ? xn[q0 + tid] : 0.f;
        tau[tid] = INFINITY;
        taui[tid] = INT_MAX;
        cnt[tid] = 0;
    }
    for (int idx = tid; idx < KQ * KCAP; idx += KNN_THREADS) { bd[idx] = INFINITY; bi[idx] = INT_MAX; }
    const int ty = tid >> 4, tx = tid & 15;   // queries ty*4 .. +3; points tx*4 .. +3 and 64 + tx*4 .. +3
    const int ntile = (n + KT - 1) / KT;
    const int t0 = q0 / KT;
    for (int tt = 0; tt < ntile; tt++) {
        const int p0 = ((t0 + tt) % ntile) * KT;
        __syncthreads();
        for (int idx = tid; idx < KT * dq; idx += KNN_THREADS) {
            const int p = idx % KT, c4 = idx / KT;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (p0 + p < n) v = *reinterpret_cast<const float4 *>(X + (size_t)(p0 + p) * dp + 4 * c4);
            ps[(4 * c4 + 0) * KT + p] = v.x;
            ps[(4 * c4 + 1) * KT + p] = v.y;
            ps[(4 * c4 + 2) * KT + p] = v.z;
            ps[(4 * c4 + 3) * KT + p] = v.w;
        }
        if (tid < KT) pn[tid] = p0 + tid < n ? xn[p0 + tid] : 0.f;
        __syncthreads();
        float acc[4][8];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
#pragma unroll 4
        for (int c = 0; c < dp; c++) {
            const float4 a = *reinterpret_cast<const float4 *>(qs + c * KQ + ty * 4);
            const float4 b0 = *reinterpret_cast<const float4 *>(ps + c * KT + tx * 4);
            const float4 b1 = *reinterpret_cast<const float4 *>(ps + c * KT + 64 + tx * 4);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = ty * 4 + i, qi = q0 + r;
            if (qi >= n) continue;
            const float th = tau[r];
            const int thi = taui[r];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int p = (j < 4 ? 0 : 64) + tx * 4 + (j & 3);
                const int gi = p0 + p;
                if (gi >= n || gi == qi) continue;
                const float d = fmaxf(fmaf(-2.f, acc[i][j], qn[r] + pn[p]), 0.f);
                if (d < th || (d == th && gi < thi)) {
                    const int slot = atomicAdd(&cnt[r], 1);
                    bd[(size_t)r * KCAP + slot] = d;
                    bi[(size_t)r * KCAP + slot] = gi;
                }
            }
        }
        __syncthreads();
        const bool last = tt == ntile - 1;
        for (int r = wid; r < KQ; r += KNN_THREADS / 32) {
            const int m = cnt[r];
            if (!(m > KBUF || (last && m > 0))) continue;
            warp_bitonic(bd + (size_t)r * KCAP, bi + (size_t)r * KCAP, lane);
            const int keep = min(m, k);
            for (int t = keep + lane; t < KCAP; t += 32) { bd[(size_t)r * KCAP + t] = INFINITY; bi[(size_t)r * KCAP + t] = INT_MAX; }
            if (lane == 0) {
                cnt[r] = keep;
                if (keep == k) { tau[r] = bd[(size_t)r * KCAP + k - 1]; taui[r] = bi[(size_t)r * KCAP + k - 1]; }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // rows re-sorted by index for the output
    for (int r = wid; r < KQ; r += KNN_THREADS / 32) {
        const int qi = q0 + r;
        if (qi >= n) continue;
        float *key = bd + (size_t)r * KCAP;
        int *tie = bi + (size_t)r * KCAP;
        for (int t = lane; t < KCAP; t += 32) {
            // sort by index: the index becomes the key (exactly representable below 2^24), the
            // squared distance rides along in the tie slot as its bits
            const int ix = tie[t];
            const float dv = key[t];
            const bool used = t < k;
            key[t] = used ? (float)ix : INFINITY;
            tie[t] = used ? __float_as_int(dv) : INT_MAX;
        }
        __syncwarp();
        warp_bitonic(key, tie, lane);
        // the reported distances by direct differences (the selection's |q|^2 + |p|^2 - 2 q.p
        // is exact enough to rank, not to report)
        for (int t = lane; t < k; t += 32) {
            const int j = (int)key[t];
            const float *xq = X + (size_t)qi * dp, *xj = X + (size_t)j * dp;
            float d2 = 0.f;
            for (int c = 0; c < dp; c += 4) {
                const float4 a4 = *reinterpret_cast<const float4 *>(xq + c);
                const float4 b4 = *reinterpret_cast<const float4 *>(xj + c);
                const float dx = a4.x - b4.x, dy = a4.y - b4.y, dz = a4.z - b4.z, dw = a4.w - b4.w;
                d2 = fmaf(dx, dx, d2); d2 = fmaf(dy, dy, d2); d2 = fmaf(dz, dz, d2); d2 = fmaf(dw, dw, d2);
            }
            out_idx[(size_t)qi * k + t] = j;
            out_d[(size_t)qi * k + t] = sqrtf(d2);
        }
        __syncwarp();
    }
}

}  // namespace

namespace tsne {

int knn_tc_run(const float *dX, int n, int dp, int dim, int k, float maxabs, int *dI, float *dD, cudaStream_t st);

// k-NN graph of the n x dim float rows of X (host, row-major) on the device: indices and
// distances (n x k each, host), rows sorted by index. 0 ok, -1 bad arguments, -2 a bounded wait
// of the tensor-core scan gave up.
int knn_graph_device(const float *X, int n, int dim, int k, int *idx_out, float *dist_out)
{
    if (X == nullptr || n < 2 || dim < 1 || k < 1 || k > n - 1 || k > KNN_WARP_MAX_K || n > (1 << 24)) return -1;
    const int dp = (dim + 3) & ~3;
    const size_t smem = knn_smem_bytes(dp);
    const bool tiled = k <= KNN_MAX_K && smem <= 227 * 1024;
    cudaStream_t st;
    TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    bool failed = false;
    const bool tm = getenv("TSNE_KNN_TIMERS") && atoi(getenv("TSNE_KNN_TIMERS")) != 0;
    auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    double t0 = now();
    {
        AllocStream guard(st);
        // centred (distances unchanged; the norms, and so the cancellation in
        // |q|^2 + |p|^2 - 2 q.p, shrink)
        // on host threads over a fixed partition of the rows (the column sums of each part are
        // added in part order, so the mean does not depend on the number of threads)
        constexpr int PARTS = 16;
        const int nth = std::max(1, std::min(PARTS, (int)std::thread::hardware_concurrency()));
        auto run_parts = [&](const std::function<void(int)> &fn) {
            std::vector<std::thread> th;
            for (int t = 1; t < nth; t++)
                th.emplace_back([&, t] { for (int part = t; part < PARTS; part += nth) fn(part); });
            for (int part = 0; part < PARTS; part += nth) fn(part);
            for (auto &x : th) x.join();
        };
        std::vector<double> psum((size_t)PARTS * dim, 0.0);
        run_parts([&](int part) {
            const int i0 = (int)((long long)n * part / PARTS), i1 = (int)((long long)n * (part + 1) / PARTS);
            double *ps = psum.data() + (size_t)part * dim;
            for (int i = i0; i < i1; i++)
                for (int c = 0; c < dim; c++) ps[c] += X[(size_t)i * dim + c];
        });
        std::vector<double> mean(dim, 0.0);
        for (int part = 0; part < PARTS; part++)
            for (int c = 0; c < dim; c++) mean[c] += psum[(size_t)part * dim + c];
        for (int c = 0; c < dim; c++) mean[c] /= n;
        std::vector<float> Xp((size_t)n * dp, 0.f), nrm(n), pmax(PARTS, 0.f);
        run_parts([&](int part) {
            const int i0 = (int)((long long)n * part / PARTS), i1 = (int)((long long)n * (part + 1) / PARTS);
            float mx = 0.f;
            for (int i = i0; i < i1; i++) {
                float s2 = 0.f;
                for (int c = 0; c < dim; c++) {
                    const float v = (float)((double)X[(size_t)i * dim + c] - mean[c]);
                    Xp[(size_t)i * dp + c] = v;
                    s2 = fmaf(v, v, s2);
                    mx = std::max(mx, std::fabs(v));
                }
                nrm[i] = s2;
            }
            pmax[part] = mx;
        });
        const float maxabs = *std::max_element(pmax.begin(), pmax.end());
        if (tm) printf("KNN host centring %.1f ms\n", 1e3 * (now() - t0));
        t0 = now();
        DevBuf<float> dX, dN, dD;
        DevBuf<int> dI;
        dX.exact(Xp.size()); dN.exact(n); dD.exact((size_t)n * k); dI.exact((size_t)n * k);
        TSNE_CUDA_CHECK(cudaMemcpyAsync(dX.p, Xp.data(), sizeof(float) * Xp.size(), cudaMemcpyHostToDevice, st));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(dN.p, nrm.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st));
        // the tensor-core scan where it applies (k <= 128, at most 64 dimensions), else the
        // CUDA-core one
        if (tm) { cudaStreamSynchronize(st); printf("KNN upload %.1f ms\n", 1e3 * (now() - t0)); t0 = now(); }
        const int tc = tiled ? knn_tc_run(dX.p, n, dp, dim, k, maxabs, dI.p, dD.p, st) : 1;
        failed = tc < 0;
        if (tc == 1 && tiled) {
            TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_knn_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_knn_tiled<<<(n + KQ - 1) / KQ, KNN_THREADS, smem, st>>>(n, dp, k, dX.p, dN.p, dI.p, dD.p);
        } else if (tc == 1) {
            // squared distances sorted by (distance, index); re-sorted by index on the host below
            k_knn_warp<<<std::min((n + 3) / 4, 148 * 32), 128, 0, st>>>(n, dp, dX.p, k, dI.p, dD.p);
        }
        TSNE_CUDA_CHECK(cudaGetLastError());
        if (tm) { cudaStreamSynchronize(st); printf("KNN scan %.1f ms\n", 1e3 * (now() - t0)); t0 = now(); }
        if (!failed) {
            TSNE_CUDA_CHECK(cudaMemcpyAsync(idx_out, dI.p, sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(dist_out, dD.p, sizeof(float) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
        }
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    cudaStreamDestroy(st);
    if (tm) printf("KNN download %.1f ms\n", 1e3 * (now() - t0));
    if (failed) return -2;
    if (!tiled) {
        std::vector<std::pair<int, float>> row(k);
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < k; j++) row[j] = {idx_out[(size_t)i * k + j], dist_out[(size_t)i * k + j]};
            std::sort(row.begin(), row.end());
            for (int j = 0; j < k; j++) {
                idx_out[(size_t)i * k + j] = row[j].first;
                dist_out[(size_t)i * k + j] = sqrtf(row[j].second);
            }
        }
    }
    return 0;
}

}  // namespace tsne

extern "C" {

int tsne_knn_graph(const float *X, int n_samples, int n_features, int k, int *indices, float *distances)
{
    if (indices == nullptr || distances == nullptr) return -1;
    try {
        return knn_graph_device(X, n_samples, n_features, k, indices, distances);
    } catch (const CudaError &) {
        return -2;
    }
}

sparse_matrix_t *compute_sparse_P(const double *X, int n_point, int pt_dim, double perplexity, int use_vptree,
                                  int verbose, int num_threads)
{
    (void)use_vptree;
    (void)num_threads;
    if (X == nullptr || n_point < 2 || pt_dim < 1 || perplexity <= 0.0) return nullptr;
    int k = (int)(3.0 * perplexity);
    if (k > n_point - 1) k = n_point - 1;
    if (k < 1 || k > KNN_WARP_MAX_K) {
        fprintf(stderr, "Error: k = %d neighbours is outside [1, %d]\n", k, KNN_WARP_MAX_K);
        return nullptr;
    }
    if (verbose) printf("Computing %d nearest neighbours on the device (exact, tiled scan)...\n", k);
    std::vector<float> Xr((size_t)n_point * pt_dim);
    for (int i = 0; i < n_point; i++)
        for (int c = 0; c < pt_dim; c++) Xr[(size_t)i * pt_dim + c] = (float)X[(size_t)c * n_point + i];
    std::vector<int> idx((size_t)n_point * k), indptr((size_t)n_point + 1);
    std::vector<float> df((size_t)n_point * k);
    try {
        if (knn_graph_device(Xr.data(), n_point, pt_dim, k, idx.data(), df.data()) != 0) return nullptr;
        std::vector<double> dist(df.begin(), df.end());
        for (int i = 0; i <= n_point; i++) indptr[i] = i * k;
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        sparse_matrix_t *P = nullptr;
        {
            AllocStream guard(st);
            DevCSR d;
            if (joint_P_device(st, n_point, dist.data(), idx.data(), indptr.data(), (long long)n_point * k,
                               perplexity, d) == 0) {
                P = sparse_matrix_create(n_point, n_point, (int)d.nnz);
                if (P != nullptr) {
                    TSNE_CUDA_CHECK(cudaMemcpyAsync(P->row_ptr, d.rp.p, sizeof(int) * ((size_t)n_point + 1),
                                                    cudaMemcpyDeviceToHost, st));
                    if (d.nnz > 0) {
                        TSNE_CUDA_CHECK(cudaMemcpyAsync(P->col_idx, d.col.p, sizeof(int) * d.nnz, cudaMemcpyDeviceToHost, st));
                        TSNE_CUDA_CHECK(cudaMemcpyAsync(P->values, d.val.p, sizeof(double) * d.nnz, cudaMemcpyDeviceToHost, st));
                    }
                    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
                    P->nnz = (int)d.nnz;
                }
            }
        }
        cudaStreamDestroy(st);
        return P;
    } catch (const CudaError &) {
        return nullptr;
    }
}

tsne_workspace_t *tsne_init(const double *X, int n_point, int pt_dim, int low_dim, const tsne_params_t *params)
{
    if (params == nullptr) return nullptr;
    if (low_dim != 2 && low_dim != 3) {
        printf("Error: low_dim must be 2 or 3 (got %d)\n", low_dim);
        return nullptr;
    }
    sparse_matrix_t *P = compute_sparse_P(X, n_point, pt_dim, params->perplexity, params->use_vptree,
                                          params->verbose, params->num_threads);
    if (P == nullptr) {
        printf("Error: Failed to compute sparse P matrix\n");
        return nullptr;
    }
    return tsne_init_with_P(X, n_point, pt_dim, low_dim, params, P);
}

int tsne_fit_transform(const double *X, int n_point, int pt_dim, int low_dim, const tsne_params_t *params,
                       double *Y_out)
{
    tsne_workspace_t *ws = tsne_init(X, n_point, pt_dim, low_dim, params);
    if (ws == nullptr) return -1;
    const int rc = tsne_run(ws);
    if (rc != 0) { tsne_destroy(ws); return rc; }
    tsne_get_embedding(ws, Y_out);
    tsne_destroy(ws);
    return 0;
}

}  // extern "C"
