// PCA initialisation and embedding quality scores on the device.
//
// tsne_pca_init: the reference's init='pca' (tsne_h2pack/manifold.py:399-416: scikit-learn's
// PCA, projection scaled to a first-coordinate standard deviation of 1e-4). Here the exact PCA:
// column means and the Gram matrix of the centred data in FP64 on the device, its symmetric
// eigen-decomposition on the host (cyclic Jacobi rotations, f x f), the projection on the
// device. Components carry scikit-learn's sign rule (each component's largest-magnitude loading
// positive, svd_flip with u_based_decision=False), so the result equals scikit-learn's exact
// PCA (svd_solver='full') to rounding; the reference's randomized solver approximates it.
//
// tsne_score_embedding: the reference's quality scores (benchmarks/quality.py:56-90): k-NN
// preservation of a set of query points (their k nearest neighbours in the embedding against
// given input-space neighbours) and the KL divergence of the embedding under a fixed P,
// sum p log p + sum p log(1 + d^2) + log Z, with Z summed over all pairs on the device (the
// reference estimates it from 1000 anchor rows).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "devbuf.h"
#include "../../include/tsne_h2pack.h"

using namespace tsne;

namespace {

constexpr int PCA_THREADS = 256;
constexpr int PCA_PAIRS = 8;                       // Gram entries per thread
constexpr int PCA_TILE_DOUBLES = 8192;             // staged rows per block: 64 KB
constexpr int PCA_ROW_BLOCKS = 148 * 2;            // fixed grid over rows (fixed summation order)

__global__ void __launch_bounds__(256) k_col_mean_part(int n, int f, const double *__restrict__ X,
                                                       double *__restrict__ part)
{
    // part[block][c]: sum over the block's rows; rows dealt in contiguous chunks per block
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int r0 = blockIdx.x * per, r1 = min(n, r0 + per);
    for (int c = threadIdx.x; c < f; c += blockDim.x) {
        double s = 0.0;
        for (int r = r0; r < r1; r++) s += X[(size_t)r * f + c];
        part[(size_t)blockIdx.x * f + c] = s;
    }
}

__global__ void k_col_mean(int n, int f, int nblk, const double *__restrict__ part, double *__restrict__ mean)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < f; c += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(size_t)b * f + c];
        mean[c] = s / n;
    }
}

// Gram partials of the centred rows: block (bx, by) takes row chunk bx and the upper-triangle
// entries by * 256 * PCA_PAIRS .. (+ 256 * PCA_PAIRS), each thread PCA_PAIRS of them
__global__ void __launch_bounds__(PCA_THREADS) k_gram_part(int n, int f, const double *__restrict__ X,
                                                           const double *__restrict__ mean, double *__restrict__ part)
{
    extern __shared__ double tile[];
    const int npair = f * (f + 1) / 2;
    const int tr = max(1, PCA_TILE_DOUBLES / f);
    int pa[PCA_PAIRS], pb[PCA_PAIRS];
    double acc[PCA_PAIRS];
#pragma unroll
    for (int q = 0; q < PCA_PAIRS; q++) {
        const int pidx = blockIdx.y * PCA_THREADS * PCA_PAIRS + q * PCA_THREADS + threadIdx.x;
        int a = -1, b = -1;
        if (pidx < npair) {   // row-major upper triangle: row a holds f - a entries
            int rem = pidx;
            a = 0;
            while (rem >= f - a) { rem -= f - a; a++; }
            b = a + rem;
        }
        pa[q] = a;
        pb[q] = b;
        acc[q] = 0.0;
    }
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int r0 = blockIdx.x * per, r1 = min(n, r0 + per);
    for (int t0 = r0; t0 < r1; t0 += tr) {
        const int cnt = min(tr, r1 - t0);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt * f; i += PCA_THREADS) tile[i] = X[(size_t)t0 * f + i] - mean[i % f];
        __syncthreads();
        for (int r = 0; r < cnt; r++) {
            const double *row = tile + (size_t)r * f;
#pragma unroll
            for (int q = 0; q < PCA_PAIRS; q++)
                if (pa[q] >= 0) acc[q] = fma(row[pa[q]], row[pb[q]], acc[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < PCA_PAIRS; q++)
        if (pa[q] >= 0) part[(size_t)blockIdx.x * npair + blockIdx.y * PCA_THREADS * PCA_PAIRS + q * PCA_THREADS +
                             threadIdx.x] = acc[q];
}

__global__ void k_gram_sum(int npair, int nblk, const double *__restrict__ part, double *__restrict__ gram)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npair; p += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; b++) s += part[(size_t)b * npair + p];
        gram[p] = s;
    }
}

// Y[i][k] = (x_i - mean) . V[:, k]
__global__ void k_project(int n, int f, int c, const double *__restrict__ X, const double *__restrict__ mean,
                          const double *__restrict__ V, double *__restrict__ Y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < c; k++) {
            double s = 0.0;
            for (int j = 0; j < f; j++) s = fma(X[(size_t)i * f + j] - mean[j], V[(size_t)j * c + k], s);
            Y[(size_t)i * c + k] = s;
        }
    }
}

// Symmetric eigen-decomposition by cyclic Jacobi rotations (the classical method, e.g. Golub
// and Van Loan, Matrix Computations, 4th ed., sec. 8.5): A (f x f, row-major) is reduced to
// diagonal form; eigenvalues in w, eigenvectors in the columns of V.
void jacobi_eigen(int f, std::vector<double> A, std::vector<double> &w, std::vector<double> &V)
{
    V.assign((size_t)f * f, 0.0);
    for (int i = 0; i < f; i++) V[(size_t)i * f + i] = 1.0;
    auto at = [&](int i, int j) -> double & { return A[(size_t)i * f + j]; };
    double total = 0.0;
    for (double x : A) total += x * x;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int i = 0; i < f; i++)
            for (int j = i + 1; j < f; j++) off += at(i, j) * at(i, j);
        if (off <= 1e-30 * total || off == 0.0) break;
        for (int p = 0; p < f; p++)
            for (int q = p + 1; q < f; q++) {
                const double apq = at(p, q);
                if (apq == 0.0) continue;
                const double theta = (at(q, q) - at(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < f; k++) {   // A <- J^T A J: columns p, q, then rows p, q
                    const double akp = at(k, p), akq = at(k, q);
                    at(k, p) = c * akp - s * akq;
                    at(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < f; k++) {
                    const double apk = at(p, k), aqk = at(q, k);
                    at(p, k) = c * apk - s * aqk;
                    at(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < f; k++) {
                    const double vkp = V[(size_t)k * f + p], vkq = V[(size_t)k * f + q];
                    V[(size_t)k * f + p] = c * vkp - s * vkq;
                    V[(size_t)k * f + q] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(f);
    for (int i = 0; i < f; i++) w[i] = at(i, i);
}

// ---- scores ----
constexpr int SCORE_KMAX = 128;

// Z = sum_{i != j} (1 + |y_i - y_j|^2)^-1 over all pairs: a thread per target, sources staged
// 256 at a time, FP32 pair terms, FP64 sums per tile, block partials in a fixed order
template <int D>
__global__ void __launch_bounds__(256) k_zexact(int n, const float *__restrict__ Y, double *__restrict__ part)
{
    __shared__ float sh[256][D];
    __shared__ double red[256];
    double Q = 0.0;
    for (int i0 = blockIdx.x * 256; i0 < n; i0 += gridDim.x * 256) {
        const int i = i0 + threadIdx.x;
        float yi[D];
        for (int k = 0; k < D; k++) yi[k] = i < n ? Y[(size_t)i * D + k] : 0.f;
        for (int base = 0; base < n; base += 256) {
            __syncthreads();
            if (base + (int)threadIdx.x < n)
                for (int k = 0; k < D; k++) sh[threadIdx.x][k] = Y[(size_t)(base + threadIdx.x) * D + k];
            __syncthreads();
            const int cnt = min(256, n - base);
            float tq = 0.f;
            for (int j = 0; j < cnt; j++) {
                float r2 = 0.f;
#pragma unroll
                for (int k = 0; k < D; k++) { const float df = yi[k] - sh[j][k]; r2 = fmaf(df, df, r2); }
                tq += (base + j == i) ? 0.f : 1.0f / (1.0f + r2);
            }
            if (i < n) Q += tq;
        }
    }
    red[threadIdx.x] = Q;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// sum p log p + sum p log(1 + d^2) over P (FP64), block partials
template <int D>
__global__ void __launch_bounds__(256) k_kl_terms(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                  const double *__restrict__ pv, const double *__restrict__ Y,
                                                  double *__restrict__ part)
{
    __shared__ double red[256];
    double t = 0.0;
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += (gridDim.x * blockDim.x) >> 5) {
        for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) {
            const int j = ci[e];
            const double p = pv[e];
            double d2 = 0.0;
            for (int k = 0; k < D; k++) { const double df = Y[(size_t)i * D + k] - Y[(size_t)j * D + k]; d2 += df * df; }
            if (p > 0.0) t += p * log(p) + p * log1p(d2);
        }
    }
    red[threadIdx.x] = t;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// k nearest embedding neighbours of each query (a warp per query, a sorted list in shared
// memory; ties keep the smaller index), then the overlap with the given input-space lists
template <int D>
__global__ void __launch_bounds__(128) k_knn_overlap(int n, const float *__restrict__ Y, int nq,
                                                     const int *__restrict__ queries, int k,
                                                     const int *__restrict__ hd, int *__restrict__ hits)
{
    __shared__ float sd[4][SCORE_KMAX];
    __shared__ int si[4][SCORE_KMAX];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *bd = sd[w];
    int *bi = si[w];
    for (int qi = blockIdx.x * 4 + w; qi < nq; qi += gridDim.x * 4) {
        const int q = queries[qi];
        for (int j = lane; j < k; j += 32) { bd[j] = INFINITY; bi[j] = INT_MAX; }
        __syncwarp();
        float yq[D];
        for (int c = 0; c < D; c++) yq[c] = Y[(size_t)q * D + c];
        for (int base = 0; base < n; base += 32) {
            const int j = base + lane;
            float d2 = INFINITY;
            if (j < n && j != q) {
                float acc = 0.f;
                for (int c = 0; c < D; c++) { const float df = yq[c] - Y[(size_t)j * D + c]; acc = fmaf(df, df, acc); }
                d2 = acc;
            }
            unsigned cand = __ballot_sync(0xffffffffu, d2 < bd[k - 1] || (d2 == bd[k - 1] && j < bi[k - 1]));
            while (cand) {
                const int src = __ffs(cand) - 1;
                cand &= cand - 1;
                const float cd = __shfl_sync(0xffffffffu, d2, src);
                const int cj = __shfl_sync(0xffffffffu, j, src);
                if (!(cd < bd[k - 1] || (cd == bd[k - 1] && cj < bi[k - 1]))) continue;
                int pos = 0;
                for (int t = lane; t < k; t += 32) pos += (bd[t] < cd || (bd[t] == cd && bi[t] < cj));
                for (int o = 16; o > 0; o >>= 1) pos += __shfl_xor_sync(0xffffffffu, pos, o);
                for (int t0 = k - 1; t0 > pos; t0 -= 32) {
                    const int t = t0 - lane;
                    float vd = 0.f;
                    int vi = 0;
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
        int h = 0;
        for (int a = lane; a < k; a += 32) {
            const int v = hd[(size_t)qi * k + a];
            for (int b = 0; b < k; b++) h += bi[b] == v;
        }
        for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
        if (lane == 0) hits[qi] = h;
        __syncwarp();
    }
}

double sum_host(const std::vector<double> &v)
{
    double s = 0.0;
    for (double x : v) s += x;
    return s;
}

}  // namespace

extern "C" {

int tsne_pca_init(const double *X, int n_samples, int n_features, int n_components, double *Y_out)
{
    if (X == nullptr || Y_out == nullptr || n_samples < 2 || n_features < 1 || n_components < 1 ||
        n_components > std::min(n_samples, n_features) || n_features > 4096) {
        fprintf(stderr, "tsne_pca_init: bad arguments (need 1 <= n_components <= min(n_samples, n_features), "
                        "n_features <= 4096)\n");
        return -1;
    }
    const int n = n_samples, f = n_features, c = n_components;
    const int npair = f * (f + 1) / 2;
    const int ny = (npair + PCA_THREADS * PCA_PAIRS - 1) / (PCA_THREADS * PCA_PAIRS);
    std::vector<double> gram_h(npair), Y((size_t)n * c);
    bool finite = true;
    try {
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        {
            AllocStream guard(st);
            DevBuf<double> dX, part, mean, gpart, gram, V, dY;
            dX.exact((size_t)n * f);
            part.exact((size_t)PCA_ROW_BLOCKS * f);
            mean.exact(f);
            gpart.exact((size_t)PCA_ROW_BLOCKS * ny * PCA_THREADS * PCA_PAIRS);
            gram.exact(npair);
            TSNE_CUDA_CHECK(cudaMemcpyAsync(dX.p, X, sizeof(double) * (size_t)n * f, cudaMemcpyHostToDevice, st));
            k_col_mean_part<<<PCA_ROW_BLOCKS, 256, 0, st>>>(n, f, dX.p, part.p);
            k_col_mean<<<(f + 255) / 256, 256, 0, st>>>(n, f, PCA_ROW_BLOCKS, part.p, mean.p);
            const int tr = std::max(1, PCA_TILE_DOUBLES / f);
            const size_t smem = sizeof(double) * (size_t)tr * f;
            TSNE_CUDA_CHECK(cudaFuncSetAttribute(k_gram_part, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_gram_part<<<dim3(PCA_ROW_BLOCKS, ny), PCA_THREADS, smem, st>>>(n, f, dX.p, mean.p, gpart.p);
            k_gram_sum<<<(npair + 255) / 256, 256, 0, st>>>(npair, PCA_ROW_BLOCKS, gpart.p, gram.p);
            TSNE_CUDA_CHECK(cudaGetLastError());
            TSNE_CUDA_CHECK(cudaMemcpyAsync(gram_h.data(), gram.p, sizeof(double) * npair, cudaMemcpyDeviceToHost, st));
            TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
            std::vector<double> A((size_t)f * f), w, Vf;
            for (int a = 0, p = 0; a < f; a++)
                for (int b = a; b < f; b++, p++) A[(size_t)a * f + b] = A[(size_t)b * f + a] = gram_h[p];
            for (double x : A) finite = finite && std::isfinite(x);
            // (the stream outlives every buffer of this scope: they are freed on it)
            if (finite) {
            jacobi_eigen(f, A, w, Vf);
            std::vector<int> ord(f);
            for (int i = 0; i < f; i++) ord[i] = i;
            std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return w[a] > w[b]; });
            std::vector<double> Vc((size_t)f * c);
            for (int k = 0; k < c; k++) {
                int big = 0;   // the largest-magnitude loading (first such) is made positive
                for (int j = 1; j < f; j++)
                    if (fabs(Vf[(size_t)j * f + ord[k]]) > fabs(Vf[(size_t)big * f + ord[k]])) big = j;
                const double sg = Vf[(size_t)big * f + ord[k]] < 0 ? -1.0 : 1.0;
                for (int j = 0; j < f; j++) Vc[(size_t)j * c + k] = sg * Vf[(size_t)j * f + ord[k]];
            }
            V.exact((size_t)f * c);
            dY.exact((size_t)n * c);
            TSNE_CUDA_CHECK(cudaMemcpyAsync(V.p, Vc.data(), sizeof(double) * Vc.size(), cudaMemcpyHostToDevice, st));
            k_project<<<148 * 8, 256, 0, st>>>(n, f, c, dX.p, mean.p, V.p, dY.p);
            TSNE_CUDA_CHECK(cudaGetLastError());
            TSNE_CUDA_CHECK(cudaMemcpyAsync(Y.data(), dY.p, sizeof(double) * Y.size(), cudaMemcpyDeviceToHost, st));
            }
            TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        }
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
        if (!finite) {
            fprintf(stderr, "tsne_pca_init: the data hold a NaN or an infinity\n");
            return -3;
        }
    } catch (const CudaError &) {
        return -2;
    }
    // the first coordinate scaled to a standard deviation of 1e-4 (population std, as numpy)
    double m0 = 0.0;
    for (int i = 0; i < n; i++) m0 += Y[(size_t)i * c];
    m0 /= n;
    double v0 = 0.0;
    for (int i = 0; i < n; i++) v0 += (Y[(size_t)i * c] - m0) * (Y[(size_t)i * c] - m0);
    const double sd = sqrt(v0 / n);
    if (!(sd > 0.0) || !std::isfinite(sd)) {
        fprintf(stderr, "tsne_pca_init: the data have no variance along the first principal component\n");
        return -3;
    }
    for (size_t i = 0; i < Y.size(); i++) Y_out[i] = Y[i] / sd * 1e-4;
    return 0;
}

int tsne_score_embedding(const double *Y, int n_point, int low_dim, const sparse_matrix_t *P, const int *queries,
                         int n_eval, const int *hd_neighbors, int k, double *knn_preservation, double *kl)
{
    if (Y == nullptr || P == nullptr || (low_dim != 2 && low_dim != 3) || n_point < 2 || P->n_rows != n_point ||
        n_eval < 0 || (n_eval > 0 && (queries == nullptr || hd_neighbors == nullptr || k < 1 || k > SCORE_KMAX ||
                                      k > n_point - 1))) {
        fprintf(stderr, "tsne_score_embedding: bad arguments\n");
        return -1;
    }
    for (int i = 0; i < n_point; i++)
        if (P->row_ptr[i] > P->row_ptr[i + 1] || P->row_ptr[0] != 0) { fprintf(stderr, "tsne_score_embedding: bad P\n"); return -1; }
    const int nnz = P->row_ptr[n_point];
    for (int e = 0; e < nnz; e++)
        if (P->col_idx[e] < 0 || P->col_idx[e] >= n_point) { fprintf(stderr, "tsne_score_embedding: bad P\n"); return -1; }
    for (int q = 0; q < n_eval; q++)
        if (queries[q] < 0 || queries[q] >= n_point) { fprintf(stderr, "tsne_score_embedding: bad query\n"); return -1; }
    // point-major copies of the embedding (FP32 for the pair sums, FP64 for the KL terms)
    const int d = low_dim, n = n_point;
    std::vector<float> yf((size_t)n * d);
    std::vector<double> yd((size_t)n * d);
    for (int i = 0; i < n; i++)
        for (int c = 0; c < d; c++) {
            yd[(size_t)i * d + c] = Y[(size_t)c * n + i];
            yf[(size_t)i * d + c] = (float)Y[(size_t)c * n + i];
        }
    constexpr int ZB = 148 * 4, KB = 148 * 8;
    std::vector<double> zp(ZB), kp(KB);
    std::vector<int> hits(std::max(n_eval, 1));
    try {
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        {
            AllocStream guard(st);
            DevBuf<float> dyf;
            DevBuf<double> dyd, dpv, dzp, dkp;
            DevBuf<int> drp, dci, dq, dhd, dhits;
            dyf.exact(yf.size()); dyd.exact(yd.size());
            drp.exact(n + 1); dci.exact(std::max(nnz, 1)); dpv.exact(std::max(nnz, 1));
            dzp.exact(ZB); dkp.exact(KB);
            TSNE_CUDA_CHECK(cudaMemcpyAsync(dyf.p, yf.data(), sizeof(float) * yf.size(), cudaMemcpyHostToDevice, st));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(dyd.p, yd.data(), sizeof(double) * yd.size(), cudaMemcpyHostToDevice, st));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(drp.p, P->row_ptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
            if (nnz > 0) {
                TSNE_CUDA_CHECK(cudaMemcpyAsync(dci.p, P->col_idx, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
                TSNE_CUDA_CHECK(cudaMemcpyAsync(dpv.p, P->values, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
            }
            if (d == 2) {
                k_zexact<2><<<ZB, 256, 0, st>>>(n, dyf.p, dzp.p);
                k_kl_terms<2><<<KB, 256, 0, st>>>(n, drp.p, dci.p, dpv.p, dyd.p, dkp.p);
            } else {
                k_zexact<3><<<ZB, 256, 0, st>>>(n, dyf.p, dzp.p);
                k_kl_terms<3><<<KB, 256, 0, st>>>(n, drp.p, dci.p, dpv.p, dyd.p, dkp.p);
            }
            if (n_eval > 0) {
                dq.exact(n_eval); dhd.exact((size_t)n_eval * k); dhits.exact(n_eval);
                TSNE_CUDA_CHECK(cudaMemcpyAsync(dq.p, queries, sizeof(int) * n_eval, cudaMemcpyHostToDevice, st));
                TSNE_CUDA_CHECK(cudaMemcpyAsync(dhd.p, hd_neighbors, sizeof(int) * (size_t)n_eval * k,
                                                cudaMemcpyHostToDevice, st));
                const int grid = std::min((n_eval + 3) / 4, 148 * 16);
                if (d == 2) k_knn_overlap<2><<<grid, 128, 0, st>>>(n, dyf.p, n_eval, dq.p, k, dhd.p, dhits.p);
                else k_knn_overlap<3><<<grid, 128, 0, st>>>(n, dyf.p, n_eval, dq.p, k, dhd.p, dhits.p);
                TSNE_CUDA_CHECK(cudaMemcpyAsync(hits.data(), dhits.p, sizeof(int) * n_eval, cudaMemcpyDeviceToHost, st));
            }
            TSNE_CUDA_CHECK(cudaGetLastError());
            TSNE_CUDA_CHECK(cudaMemcpyAsync(zp.data(), dzp.p, sizeof(double) * ZB, cudaMemcpyDeviceToHost, st));
            TSNE_CUDA_CHECK(cudaMemcpyAsync(kp.data(), dkp.p, sizeof(double) * KB, cudaMemcpyDeviceToHost, st));
            TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        }
        cudaStreamDestroy(st);
    } catch (const CudaError &) {
        return -2;
    }
    const double Z = sum_host(zp);
    if (kl) *kl = sum_host(kp) + log(Z);
    if (knn_preservation) {
        long long h = 0;
        for (int q = 0; q < n_eval; q++) h += hits[q];
        *knn_preservation = n_eval > 0 ? (double)h / ((double)n_eval * k) : 0.0;
    }
    return 0;
}

}  // extern "C"
