// The joint probabilities P on the device: the reference's conditional calibration
// (src/tsne_utils.c:1022-1105, device FP64 bisection in dense.cu) followed by the
// symmetrisation and normalisation that its Python layer does on the host
// (tsne_h2pack/_backend.py:709-718: P = (P_c + P_c^T) / sum, scipy's csr addition).
//
// Symmetrisation as one sort: every entry (i, j, p) of P_c is written twice, under the keys
// i n + j and j n + i; a stable radix sort brings the (at most two) contributions to each
// (row, column) together, in row-major order; each key's sum is its first value plus, when
// the next entry holds the same key, that value (a + b is commutative in IEEE arithmetic, so
// the sum equals scipy's bit for bit). Sums that are exactly zero are dropped, as scipy's
// addition drops them. The normalising total is a fixed-order FP64 sum (the same bits on every
// run; it differs from numpy's pairwise sum by rounding only).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <cub/cub.cuh>

#include "common.cuh"
#include "devbuf.h"
#include "kernels.h"
#include "pjoint.h"
#include "../../include/tsne_h2pack.h"

namespace tsne {

namespace {

constexpr int SUM_BLOCKS = 148 * 4;

// rows strictly increasing by column, no self entry, columns in [0, n) (row pointers already
// checked on the host)
__global__ void k_knn_check(int n, const int *__restrict__ rp, const int *__restrict__ ci, int *__restrict__ bad)
{
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        const int b = rp[i], e = rp[i + 1];
        for (int k = b + lane; k < e; k += 32) {
            const int c = ci[k];
            if (c < 0 || c >= n || c == i || (k > b && ci[k - 1] >= c)) atomicExch(bad, 1);
        }
    }
}

// entry k of row i (column j, value p) -> keys i n + j and j n + i at 2k, 2k + 1
__global__ void k_sym_keys(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                           const double *__restrict__ pv, unsigned long long *__restrict__ keys,
                           double *__restrict__ vals)
{
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        const int b = rp[i], e = rp[i + 1];
        for (int k = b + lane; k < e; k += 32) {
            const unsigned long long j = (unsigned)ci[k];
            const double p = pv[k];
            keys[2 * (size_t)k] = (unsigned long long)i * n + j;
            keys[2 * (size_t)k + 1] = j * n + (unsigned long long)i;
            vals[2 * (size_t)k] = p;
            vals[2 * (size_t)k + 1] = p;
        }
    }
}

// keep[s] = 1 where s starts a run of equal keys and the run's sum is not zero
__global__ void k_sym_keep(long long m, const unsigned long long *__restrict__ keys, const double *__restrict__ vals,
                           int *__restrict__ keep)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m; s += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[s];
        int f = 0;
        if (s == 0 || keys[s - 1] != k) {
            const double v = vals[s] + ((s + 1 < m && keys[s + 1] == k) ? vals[s + 1] : 0.0);
            f = v != 0.0;
        }
        keep[s] = f;
    }
}

__global__ void k_sym_compact(long long m, int n, const unsigned long long *__restrict__ keys,
                              const double *__restrict__ vals, const int *__restrict__ keep,
                              const int *__restrict__ pos, int *__restrict__ col, double *__restrict__ val,
                              int *__restrict__ row)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < m; s += (long long)gridDim.x * blockDim.x) {
        if (!keep[s]) continue;
        const unsigned long long k = keys[s];
        const int u = pos[s];
        row[u] = (int)(k / (unsigned long long)n);
        col[u] = (int)(k % (unsigned long long)n);
        val[u] = vals[s] + ((s + 1 < m && keys[s + 1] == k) ? vals[s + 1] : 0.0);
    }
}

// row pointers from the rows of the kept entries (sorted): row_ptr[r] = first u with row >= r
__global__ void k_sym_rowptr(int cnt, int n, const int *__restrict__ row, int *__restrict__ rp)
{
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u <= cnt; u += (long long)gridDim.x * blockDim.x) {
        const int lo = u == 0 ? -1 : row[u - 1];
        const int hi = u == cnt ? n : row[u];
        for (int r = lo + 1; r <= hi; r++) rp[r] = (int)u;
    }
}

// fixed-order FP64 sum: block partials over a fixed grid, then every block of the scaling
// kernel sums the partials in the same order
__global__ void __launch_bounds__(256) k_sum_part(int cnt, const double *__restrict__ val, double *__restrict__ part)
{
    __shared__ double sh[256];
    double t = 0.0;
    for (int u = blockIdx.x * 256 + threadIdx.x; u < cnt; u += gridDim.x * 256) t += val[u];
    sh[threadIdx.x] = t;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(256) k_scale(int cnt, double *__restrict__ val, const double *__restrict__ part,
                                               int nblk, double *__restrict__ total_out)
{
    __shared__ double sh[256];
    double t = 0.0;
    for (int b = threadIdx.x; b < nblk; b += 256) t += part[b];
    sh[threadIdx.x] = t;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const double total = sh[0];
    if (blockIdx.x == 0 && threadIdx.x == 0 && total_out != nullptr) *total_out = total;
    if (!(total > 0.0)) return;
    for (int u = blockIdx.x * 256 + threadIdx.x; u < cnt; u += gridDim.x * 256) val[u] = val[u] / total;
}

int key_bits(int n)
{
    const unsigned long long top = (unsigned long long)n * (unsigned long long)n;
    int b = 1;
    while (b < 64 && (1ULL << b) < top) b++;
    return b;
}

}  // namespace

int joint_P_device(cudaStream_t st, int n, const double *knn_dist, const int *knn_ind, const int *knn_indptr,
                   long long nnz, double perplexity, DevCSR &out)
{
    if (n < 1 || nnz < 0 || !(perplexity > 0.0)) return -1;
    if (2 * nnz > 0x7fffffffLL) {
        fprintf(stderr, "tsne_h2pack: the k-NN graph has %lld entries; the device P construction takes at most %lld\n",
                nnz, 0x7fffffffLL / 2);
        return -1;
    }
    out.n = n;
    out.rp.exact((size_t)n + 1);
    if (nnz == 0) {
        TSNE_CUDA_CHECK(cudaMemsetAsync(out.rp.p, 0, sizeof(int) * ((size_t)n + 1), st));
        out.nnz = 0;
        return 0;
    }
    const long long m = 2 * nnz;
    DevBuf<unsigned long long> keys, keys2;
    DevBuf<double> vals, vals2;
    DevBuf<int> flag;
    {
        DevBuf<int> ip, ci;
        DevBuf<double> dist, pc;
        ip.exact((size_t)n + 1);
        ci.exact(nnz);
        dist.exact(nnz);
        pc.exact(nnz);
        flag.exact(1);
        // row pointers checked on the host before the device reads through them
        bool rows_ok = knn_indptr[0] == 0 && knn_indptr[n] == nnz;
        for (int i = 0; rows_ok && i < n; i++) rows_ok = knn_indptr[i] <= knn_indptr[i + 1];
        if (!rows_ok) {
            fprintf(stderr, "tsne_h2pack: k-NN row pointers must run from 0 to nnz without decreasing\n");
            return -1;
        }
        TSNE_CUDA_CHECK(cudaMemcpyAsync(ip.p, knn_indptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, st));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(ci.p, knn_ind, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(dist.p, knn_dist, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
        TSNE_CUDA_CHECK(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
        k_knn_check<<<148 * 8, 256, 0, st>>>(n, ip.p, ci.p, flag.p);
        int bad = 0;
        TSNE_CUDA_CHECK(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        if (bad) {
            fprintf(stderr, "tsne_h2pack: k-NN rows must be sorted by column, without self entries, with columns "
                            "in [0, n)\n");
            return -1;
        }
        launch_pcal(st, n, ip.p, dist.p, perplexity, pc.p);
        keys.exact(m);
        vals.exact(m);
        k_sym_keys<<<148 * 8, 256, 0, st>>>(n, ip.p, ci.p, pc.p, keys.p, vals.p);
    }
    keys2.exact(m);
    vals2.exact(m);
    {
        size_t bytes = 0;
        TSNE_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.p, keys2.p, vals.p, vals2.p, (int)m, 0,
                                                        key_bits(n), st));
        DevBuf<unsigned char> tmp;
        tmp.exact(bytes + 256);
        TSNE_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, keys.p, keys2.p, vals.p, vals2.p, (int)m, 0,
                                                        key_bits(n), st));
    }
    keys.release();
    vals.release();
    DevBuf<int> keep, pos;
    keep.exact(m + 1);
    pos.exact(m + 1);
    k_sym_keep<<<148 * 8, 256, 0, st>>>(m, keys2.p, vals2.p, keep.p);
    TSNE_CUDA_CHECK(cudaMemsetAsync(keep.p + m, 0, sizeof(int), st));
    {
        size_t bytes = 0;
        TSNE_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, keep.p, pos.p, (int)(m + 1), st));
        DevBuf<unsigned char> tmp;
        tmp.exact(bytes + 256);
        TSNE_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, keep.p, pos.p, (int)(m + 1), st));
    }
    int cnt = 0;
    TSNE_CUDA_CHECK(cudaMemcpyAsync(&cnt, pos.p + m, sizeof(int), cudaMemcpyDeviceToHost, st));
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    out.col.exact(std::max(cnt, 1));
    out.val.exact(std::max(cnt, 1));
    DevBuf<int> row;
    row.exact(std::max(cnt, 1));
    k_sym_compact<<<148 * 8, 256, 0, st>>>(m, n, keys2.p, vals2.p, keep.p, pos.p, out.col.p, out.val.p, row.p);
    k_sym_rowptr<<<148 * 8, 256, 0, st>>>(cnt, n, row.p, out.rp.p);
    DevBuf<double> part, total;
    part.exact(SUM_BLOCKS);
    total.exact(1);
    k_sum_part<<<SUM_BLOCKS, 256, 0, st>>>(cnt, out.val.p, part.p);
    k_scale<<<SUM_BLOCKS, 256, 0, st>>>(cnt, out.val.p, part.p, SUM_BLOCKS, total.p);
    TSNE_CUDA_CHECK(cudaGetLastError());
    out.nnz = cnt;
    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace tsne

using namespace tsne;

extern "C" TSNE_API sparse_matrix_t *tsne_joint_P_from_knn_distances(const double *knn_distances,
                                                                     const int *knn_indices, const int *knn_indptr,
                                                                     int n_samples, int nnz, double perplexity)
{
    if (knn_indptr == nullptr || n_samples < 1 || nnz < 0 || (nnz > 0 && (knn_distances == nullptr ||
                                                                          knn_indices == nullptr)))
        return nullptr;
    try {
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        sparse_matrix_t *P = nullptr;
        {
            AllocStream guard(st);
            DevCSR d;
            if (joint_P_device(st, n_samples, knn_distances, knn_indices, knn_indptr, nnz, perplexity, d) == 0) {
                P = sparse_matrix_create(n_samples, n_samples, (int)d.nnz);
                if (P != nullptr) {
                    TSNE_CUDA_CHECK(cudaMemcpyAsync(P->row_ptr, d.rp.p, sizeof(int) * ((size_t)n_samples + 1),
                                                    cudaMemcpyDeviceToHost, st));
                    if (d.nnz > 0) {
                        TSNE_CUDA_CHECK(cudaMemcpyAsync(P->col_idx, d.col.p, sizeof(int) * d.nnz,
                                                        cudaMemcpyDeviceToHost, st));
                        TSNE_CUDA_CHECK(cudaMemcpyAsync(P->values, d.val.p, sizeof(double) * d.nnz,
                                                        cudaMemcpyDeviceToHost, st));
                    }
                    TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
                    P->nnz = (int)d.nnz;
                }
            }
        }
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
        return P;
    } catch (const CudaError &) {
        return nullptr;
    }
}
