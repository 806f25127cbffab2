"""Seeded synthetic workloads (Gaussian mixtures) standing in for the benchmark datasets.

The reference benchmarks on the Zheng 10x mouse-brain cells (1.3M x 50 PCA dims), a
shared k=90 neighbour graph, perplexity 30. These generators reproduce that shape with
seeded Gaussian mixtures; the graph is built once, outside any timed region.
"""
import numpy as np


def mixture_equal(n, n_clusters=10, dim=50, center_std=5.0, seed=0, dtype=np.float64):
    """n points in `n_clusters` equal clusters, centres ~ N(0, center_std^2 I), unit noise."""
    rng = np.random.default_rng(seed)
    centers = rng.normal(0.0, center_std, (n_clusters, dim))
    lab = np.repeat(np.arange(n_clusters), -(-n // n_clusters))[:n]
    X = centers[lab] + rng.standard_normal((n, dim))
    return X.astype(dtype), lab


def mixture_zipf(n, n_clusters=100, dim=50, s=1.1, seed=1, dtype=np.float32):
    """Zipf(s)-sized clusters, centres ~ N(0, 3^2 I), per-dimension std ~ U(0.5, 2)."""
    rng = np.random.default_rng(seed)
    w = np.arange(1, n_clusters + 1, dtype=np.float64) ** (-s)
    counts = rng.multinomial(n, w / w.sum())
    centers = rng.normal(0.0, 3.0, (n_clusters, dim))
    sd = rng.uniform(0.5, 2.0, (n_clusters, dim))
    lab = np.repeat(np.arange(n_clusters), counts)
    X = centers[lab] + sd[lab] * rng.standard_normal((n, dim))
    return X.astype(dtype), lab


def knn_graph(X, k, n_jobs=-1):
    """Exact k-NN distance graph (CSR, L2 distances, self excluded) on the host."""
    from sklearn.neighbors import NearestNeighbors
    nn = NearestNeighbors(n_neighbors=k, algorithm="brute", n_jobs=n_jobs).fit(X)
    return nn.kneighbors_graph(mode="distance")


def knn_graph_torch(X, k, device="cuda", chunk=8192):
    """Exact k-NN distance graph computed with torch on a GPU (harness only: builds the
    benchmark's shared input graph once, outside every timed region)."""
    import torch
    from scipy.sparse import csr_matrix
    n = X.shape[0]
    Xt = torch.as_tensor(np.ascontiguousarray(X), dtype=torch.float32, device=device)
    sq = (Xt * Xt).sum(1)
    idx_all = np.empty((n, k), dtype=np.int32)
    dst_all = np.empty((n, k), dtype=np.float64)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        d2 = sq[s:e, None] + sq[None, :] - 2.0 * (Xt[s:e] @ Xt.T)
        d2[torch.arange(e - s, device=device), torch.arange(s, e, device=device)] = float("inf")
        val, idx = torch.topk(d2, k, dim=1, largest=False)
        dst_all[s:e] = val.clamp_min(0).sqrt().double().cpu().numpy()
        idx_all[s:e] = idx.int().cpu().numpy()
    indptr = np.arange(0, (n + 1) * k, k, dtype=np.int64)
    G = csr_matrix((dst_all.ravel(), idx_all.ravel(), indptr), shape=(n, n))
    G.sort_indices()
    return G


def symmetric_P(P_cond):
    """P = (P_cond + P_cond^T) / sum, as the reference's backend does after calibration."""
    Ps = P_cond + P_cond.T
    total = Ps.sum()
    if total > 0:
        Ps.data /= total
    Ps.sort_indices()
    return Ps.tocsr()
