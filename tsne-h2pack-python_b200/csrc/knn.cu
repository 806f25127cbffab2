// Legacy feature-space entry points of the C ABI: compute_sparse_P (reference
// src/tsne_utils.c:828-933, there a ball-tree k-NN on the host), tsne_init and
// tsne_fit_transform. Here the exact k nearest neighbours (k = 3 * perplexity) are found by a
// brute-force device scan, the conditional P by the device beta bisection, and P is
// symmetrised as P + P^T and normalised, as the reference's Python backend does
// (tsne_h2pack/_backend.py:709-718).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <utility>
#include <vector>

#include "common.cuh"
#include "devbuf.h"
#include "kernels.h"
#include "../../include/tsne_h2pack.h"

using namespace tsne;

namespace {

constexpr int KNN_MAX_K = 256;

// One warp per query: distances to every point in chunks of 32, a sorted top-k list in
// shared memory updated by warp-cooperative insertion. Ties keep the smaller index.
__global__ void __launch_bounds__(128)
k_knn(int n, int dim, const float *__restrict__ X, int k, int *__restrict__ out_idx, float *__restrict__ out_d2)
{
    __shared__ float sd[4][KNN_MAX_K];
    __shared__ int si[4][KNN_MAX_K];
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

}  // namespace

extern "C" {

sparse_matrix_t *compute_sparse_P(const double *X, int n_point, int pt_dim, double perplexity, int use_vptree,
                                  int verbose, int num_threads)
{
    (void)use_vptree;
    if (X == nullptr || n_point < 2 || pt_dim < 1 || perplexity <= 0.0) return nullptr;
    int k = (int)(3.0 * perplexity);
    if (k > n_point - 1) k = n_point - 1;
    if (k < 1 || k > KNN_MAX_K) {
        fprintf(stderr, "Error: k = %d neighbours is outside [1, %d]\n", k, KNN_MAX_K);
        return nullptr;
    }
    if (verbose) printf("Computing %d nearest neighbours on the device (brute force)...\n", k);
    std::vector<float> Xr((size_t)n_point * pt_dim);
    for (int i = 0; i < n_point; i++)
        for (int c = 0; c < pt_dim; c++) Xr[(size_t)i * pt_dim + c] = (float)X[(size_t)c * n_point + i];
    std::vector<int> idx((size_t)n_point * k);
    std::vector<float> d2((size_t)n_point * k);
    try {
        cudaStream_t st;
        TSNE_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DevBuf<float> dX, dD;
        DevBuf<int> dI;
        dX.exact(Xr.size()); dD.exact(d2.size()); dI.exact(idx.size());
        TSNE_CUDA_CHECK(cudaMemcpyAsync(dX.p, Xr.data(), sizeof(float) * Xr.size(), cudaMemcpyHostToDevice, st));
        k_knn<<<std::min(ceil_div(n_point, 4), 148 * 32), 128, 0, st>>>(n_point, pt_dim, dX.p, k, dI.p, dD.p);
        TSNE_CUDA_CHECK(cudaGetLastError());
        TSNE_CUDA_CHECK(cudaMemcpyAsync(idx.data(), dI.p, sizeof(int) * idx.size(), cudaMemcpyDeviceToHost, st));
        TSNE_CUDA_CHECK(cudaMemcpyAsync(d2.data(), dD.p, sizeof(float) * d2.size(), cudaMemcpyDeviceToHost, st));
        TSNE_CUDA_CHECK(cudaStreamSynchronize(st));
        cudaStreamDestroy(st);
    } catch (const CudaError &) {
        return nullptr;
    }
    // rows sorted by column, as the reference backend hands them to the calibration
    std::vector<int> indptr(n_point + 1), ind((size_t)n_point * k);
    std::vector<double> dist((size_t)n_point * k);
    std::vector<std::pair<int, float>> row(k);
    for (int i = 0; i < n_point; i++) {
        for (int j = 0; j < k; j++) row[j] = {idx[(size_t)i * k + j], d2[(size_t)i * k + j]};
        std::sort(row.begin(), row.end());
        for (int j = 0; j < k; j++) {
            ind[(size_t)i * k + j] = row[j].first;
            dist[(size_t)i * k + j] = sqrt((double)row[j].second);
        }
        indptr[i] = i * k;
    }
    indptr[n_point] = n_point * k;
    sparse_matrix_t *Pc = compute_P_from_knn_distances(dist.data(), ind.data(), indptr.data(), n_point, n_point * k,
                                                       perplexity, num_threads);
    if (Pc == nullptr) return nullptr;
    // P = (Pc + Pc^T) / sum
    std::vector<int> cnt(n_point + 1, 0);
    for (int i = 0; i < n_point; i++)
        for (int e = Pc->row_ptr[i]; e < Pc->row_ptr[i + 1]; e++) { cnt[i]++; cnt[Pc->col_idx[e]]++; }
    std::vector<int> start(n_point + 1, 0);
    for (int i = 0; i < n_point; i++) start[i + 1] = start[i] + cnt[i];
    std::vector<std::pair<int, double>> ent(start[n_point]);
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < n_point; i++)
        for (int e = Pc->row_ptr[i]; e < Pc->row_ptr[i + 1]; e++) {
            const int j = Pc->col_idx[e];
            ent[fill[i]++] = {j, Pc->values[e]};
            ent[fill[j]++] = {i, Pc->values[e]};
        }
    sparse_matrix_destroy(Pc);
    std::vector<int> rp(n_point + 1, 0), ci;
    std::vector<double> pv;
    ci.reserve(ent.size());
    pv.reserve(ent.size());
    double total = 0.0;
    for (int i = 0; i < n_point; i++) {
        std::sort(ent.begin() + start[i], ent.begin() + start[i + 1],
                  [](const std::pair<int, double> &a, const std::pair<int, double> &b) { return a.first < b.first; });
        for (int e = start[i]; e < start[i + 1]; e++) {
            if (!ci.empty() && (int)ci.size() > rp[i] && ci.back() == ent[e].first) pv.back() += ent[e].second;
            else { ci.push_back(ent[e].first); pv.push_back(ent[e].second); }
        }
        rp[i + 1] = (int)ci.size();
    }
    for (double x : pv) total += x;
    sparse_matrix_t *P = sparse_matrix_create(n_point, n_point, (int)ci.size());
    if (P == nullptr) return nullptr;
    memcpy(P->row_ptr, rp.data(), sizeof(int) * (n_point + 1));
    memcpy(P->col_idx, ci.data(), sizeof(int) * ci.size());
    for (size_t e = 0; e < pv.size(); e++) P->values[e] = total > 0 ? pv[e] / total : pv[e];
    return P;
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
