"""PCA initialisation and quality scores on the device (tsne_pca_init, tsne_score_embedding):

  - init='pca': equals scikit-learn's exact PCA (svd_solver='full', its sign rule) scaled to a
    first-coordinate std of 1e-4, to rel 1e-9; within 2e-3 of the reference's randomized PCA
    (its own approximation error) on the benchmark mixture; non-finite or constant data raise;
  - scores: KL under a fixed P with the exact Z, against the FP64 host sum over all pairs
    (rel 1e-6; the device sums single-precision pair terms in double), and k-NN preservation
    against the host computation of the reference's benchmarks/quality.py (KD-tree
    neighbours), to 1e-3 (ties of single-precision distances aside).
"""
import numpy as np
import pytest

import oracle as O
from helpers import problem

pytestmark = pytest.mark.gpu


def _be():
    from tsne_h2pack._backend import get_backend
    return get_backend()


def _sk_pca(X, c, solver="full", rs=0):
    from sklearn.decomposition import PCA
    Y = PCA(n_components=c, svd_solver=solver, random_state=rs).fit_transform(np.asarray(X, dtype=np.float64))
    return Y / np.std(Y[:, 0]) * 1e-4


@pytest.mark.parametrize("n,f,c", [(5000, 50, 2), (3001, 7, 3), (2000, 300, 2)])
def test_pca_init_equals_exact_pca(n, f, c):
    rng = np.random.default_rng(n + f)
    X = rng.normal(size=(n, f)) @ rng.normal(size=(f, f)) + rng.normal(3.0, 1.0, size=f)
    Y = _be().pca_init(X, c)
    Ye = _sk_pca(X, c)
    assert np.abs(Y - Ye).max() <= 1e-9 * np.abs(Ye).max()


def test_pca_init_near_reference_randomized_pca():
    from tsne_h2pack._synthetic import mixture_zipf
    X, _ = mixture_zipf(50_000, seed=1)
    Y = _be().pca_init(X.astype(np.float64), 2)
    Yr = _sk_pca(X, 2, solver="randomized", rs=0)
    assert np.abs(Y - Yr).max() <= 2e-3 * np.abs(Yr).max()


def test_pca_init_bad_data_raise():
    X = np.random.default_rng(0).normal(size=(500, 10))
    X[3, 4] = np.nan
    with pytest.raises(ValueError):
        _be().pca_init(X, 2)
    with pytest.raises(ValueError):
        _be().pca_init(np.ones((500, 10)), 2)


def _host_scores(Y, P, G, k, queries):
    from sklearn.neighbors import KDTree
    n = Y.shape[0]
    ld = KDTree(Y).query(Y[queries], k=k + 1, return_distance=False)[:, 1:]
    hits = 0
    for r, i in enumerate(queries):
        a, b = G.indptr[i], G.indptr[i + 1]
        hd = G.indices[a:b][np.argsort(G.data[a:b], kind="stable")[:k]]
        hits += len(set(hd.tolist()) & set(ld[r].tolist()))
    P = P.tocsr()
    rows = np.repeat(np.arange(n), np.diff(P.indptr))
    d2 = ((Y[rows] - Y[P.indices]) ** 2).sum(1)
    Z = 0.0
    for s in range(0, n, 500):
        r2 = ((Y[s:s + 500, None, :] - Y[None, :, :]) ** 2).sum(-1)
        w = 1.0 / (1.0 + r2)
        Z += w.sum() - min(500, n - s)
    p = P.data
    kl = float(np.sum(p * np.log(p)) + np.sum(p * np.log1p(d2)) + np.log(Z))
    return hits / (k * len(queries)), kl


@pytest.mark.parametrize("d", [2, 3])
def test_scores_match_host(d):
    X, G, P, _ = problem(6000, seed=4, dim=20)
    Y0 = O.init_embedding(P.shape[0], d, 2)
    Y, _ = O.run(P, Y0, n_iter=200) if d == 2 else (Y0 * 1e4, None)
    Yp = np.ascontiguousarray(Y.T)
    out = _be().score_embedding(Yp, P, G, k=10, n_eval=2000, seed=1)
    q = np.random.default_rng(1).choice(P.shape[0], size=2000, replace=False)
    kp, kl = _host_scores(Yp, P, G.tocsr(), 10, q)
    assert abs(out["kl"] - kl) <= 1e-6 * abs(kl)
    assert abs(out["knn_preservation"] - kp) <= 1e-3
