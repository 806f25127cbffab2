"""The device k-NN graph (tsne_knn_graph, knn_method='cuda') against exact FP64 neighbours
(the graph the reference's knn_method='exact' builds with scikit-learn's brute force):

  - every returned neighbour is within the true k-th distance (FP64) up to the selection's
    single-precision rounding (rel 1e-5), and the index sets equal the exact ones on >= 99% of
    the rows (the rest differ only at distances that tie to that rounding);
  - distances within 1e-5 relative of the FP64 distances of the same pairs;
  - rows sorted by index, self excluded;
  - sizes that are not multiples of the tiles, dimensions not a multiple of 4, k above the
    tiled scan's limit (the per-query kernel), and duplicate points (found at distance 0).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_graph(X, k):
    from tsne_h2pack._knn_methods import get_knn_method
    G = get_knn_method("cuda").compute(X, k)
    n = X.shape[0]
    return G.indices.reshape(n, k), G.data.reshape(n, k)


def _exact(X, k):
    from sklearn.neighbors import NearestNeighbors
    X64 = np.asarray(X, dtype=np.float64)
    d, i = NearestNeighbors(n_neighbors=k + 1, algorithm="brute").fit(X64).kneighbors(X64)
    return d, i


@pytest.mark.parametrize("n,dim,k", [(5000, 50, 90), (3001, 7, 30), (1500, 33, 150), (20000, 50, 45)])
def test_device_knn_matches_exact(n, dim, k):
    rng = np.random.default_rng(n + dim)
    centres = rng.normal(0, 3, size=(12, dim))
    X = (centres[rng.integers(0, 12, n)] + rng.uniform(0.5, 2.0, size=(12, dim))[rng.integers(0, 12, n)]
         * rng.standard_normal((n, dim))).astype(np.float32)
    X[10] = X[20]                                   # a duplicate pair
    idx, dist = _device_graph(X, k)
    assert np.all(np.diff(idx, axis=1) > 0)         # sorted by index, no repeats
    assert not np.any(idx == np.arange(n)[:, None])
    d_ex, i_ex = _exact(X, k)
    X64 = X.astype(np.float64)
    true_d = np.sqrt(((X64[:, None, :] - X64[idx]) ** 2).sum(-1)) if n <= 5000 else None
    same = 0
    for r in range(n):
        ex = i_ex[r][i_ex[r] != r][:k]
        if set(ex.tolist()) == set(idx[r].tolist()):
            same += 1
        # the k-th true distance bounds every returned neighbour's true distance
        dk = np.sort(np.linalg.norm(X64[ex] - X64[r], axis=1))[-1]
        dr = np.linalg.norm(X64[idx[r]] - X64[r], axis=1)
        assert dr.max() <= dk * (1 + 1e-5) + 1e-6, r
        np.testing.assert_allclose(dist[r], dr, rtol=1e-5, atol=1e-5)
    assert same >= 0.99 * n, same
    assert 20 in idx[10] and 10 in idx[20]
    if true_d is not None:
        np.testing.assert_allclose(dist, true_d, rtol=1e-5, atol=1e-5)
