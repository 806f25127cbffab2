"""The Python host layer (parameter validation and mapping onto tsne_params_t); no GPU."""
import numpy as np
import pytest

from tsne_h2pack import H2_DEFAULTS, TSNE, h2_defaults
from tsne_h2pack.manifold import _resolve_n_jobs


def test_h2_defaults_per_dimension():
    assert h2_defaults(2) == dict(h2_tol=1e-2, h2_rebuild_freq=3, h2_rebuild_freq_early=10, h2_leaf_size=100)
    assert h2_defaults(3)["h2_tol"] == 3e-2 and h2_defaults(5) == H2_DEFAULTS[3]
    t = TSNE(n_components=3)
    assert t.h2_tol == 3e-2 and t.h2_rebuild_freq == 3


@pytest.mark.parametrize("kw", [dict(metric="cosine"), dict(init="spectral"), dict(method="bh"),
                                dict(n_components=0), dict(perplexity=0), dict(learning_rate="fast"),
                                dict(learning_rate=-1.0), dict(h2_rebuild_freq=0), dict(h2_leaf_size=0),
                                dict(max_iter=0), dict(init=np.zeros((5, 3)))])
def test_invalid_parameters_raise(kw):
    with pytest.raises(ValueError):
        TSNE(**kw)


def test_param_mapping():
    t = TSNE(method="exact", learning_rate="auto", h2_rebuild_freq_early=2, random_state=7, n_jobs=-1)
    p = t._map_params_to_c_struct(n_samples=24000)
    assert p.h2_rebuild_freq == 999999 and p.h2_tol == 1e-4
    assert p.learning_rate == 2000.0
    assert p.h2_rebuild_freq_early == 3         # never below the late frequency
    assert p.random_seed == 7 and p.num_threads >= 1
    p2 = TSNE(learning_rate=350.0)._map_params_to_c_struct(n_samples=100)
    assert p2.learning_rate == 350.0 and p2.h2_rebuild_freq == 3 and p2.sklearn_compatible == 1


def test_resolve_n_jobs():
    import os
    assert _resolve_n_jobs(None) == 1 and _resolve_n_jobs(0) == 1 and _resolve_n_jobs(4) == 4
    assert _resolve_n_jobs(-1) == max(1, os.cpu_count() or 1)


def test_validate_data():
    t = TSNE(perplexity=30)
    with pytest.raises(ValueError):
        t._validate_data(np.zeros(5))
    with pytest.raises(ValueError):
        t._validate_data(np.zeros((10, 3)))          # perplexity >= n_samples
    with pytest.raises(ValueError):
        t._validate_data(np.full((100, 3), np.nan))


def test_precomputed_graph_checks():
    from scipy.sparse import csr_matrix
    t = TSNE(metric="precomputed", perplexity=5, init="random")
    with pytest.raises(ValueError):
        t.fit_transform(np.zeros((10, 10)))          # dense
    with pytest.raises(ValueError):
        t.fit_transform(csr_matrix(np.ones((10, 12))))
    G = csr_matrix(np.ones((10, 10)) - np.eye(10))
    with pytest.raises(ValueError):
        TSNE(metric="precomputed", perplexity=9, init="random").fit_transform(G)   # 9 neighbours <= 9
    with pytest.raises(ValueError):
        t.fit_transform(csr_matrix(-(np.ones((10, 10)) - np.eye(10))))            # negative distances


def test_no_cpu_fallback_without_a_device():
    """Without a CUDA device the engine's calls fail and TSNE raises: nothing on the path
    falls back to the CPU."""
    import torch
    from helpers import problem
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    X, G, P, _ = problem(300, seed=0, k=30, perplexity=10.0, dim=8, n_clusters=3)
    with pytest.raises(RuntimeError):
        TSNE(metric="precomputed", perplexity=10, max_iter=10, init="random").fit_transform(G)


def test_prepare_knn_graph_drops_self_entries_and_sorts():
    """The graph handed to the device calibration: rows sorted by column, self entries dropped,
    for k-NN graphs (k entries in every row) and ragged graphs alike; a k-NN graph without
    self entries passes through unchanged."""
    from scipy.sparse import csr_matrix
    from tsne_h2pack._backend import TSNEBackend
    prep = TSNEBackend.prepare_knn_graph
    rng = np.random.default_rng(3)
    n, k = 50, 6
    idx = np.stack([rng.choice(np.delete(np.arange(n), i), k, replace=False) for i in range(n)]).astype(np.int32)
    dist = rng.random((n, k)) + 0.1
    G = csr_matrix((dist.ravel(), idx.ravel(), np.arange(0, (n + 1) * k, k)), shape=(n, n))
    G.sort_indices()
    assert prep(G) is G
    # unsorted rows with self entries in rows 3 and 17
    idx2 = idx.copy()
    idx2[3, 2], idx2[17, 0] = 3, 17
    G2 = csr_matrix((dist.ravel(), idx2.ravel(), np.arange(0, (n + 1) * k, k)), shape=(n, n))
    out = prep(G2)
    assert out.has_sorted_indices and out.nnz == n * k - 2
    dense_in, dense_out = G2.toarray(), out.toarray()
    np.fill_diagonal(dense_in, 0.0)
    np.testing.assert_array_equal(dense_out, dense_in)
    # ragged rows: the general path
    G3 = G2.tolil()
    G3[5, [c for c in range(n) if G3[5, c] != 0][:2]] = 0
    G3 = csr_matrix(G3)
    G3.eliminate_zeros()
    out3 = prep(G3)
    d3 = G3.toarray()
    np.fill_diagonal(d3, 0.0)
    np.testing.assert_array_equal(out3.toarray(), d3)
    assert not np.any(out3.indices == np.repeat(np.arange(n), np.diff(out3.indptr)))


def test_feature_path_hands_float32_to_the_device_knn(monkeypatch):
    """knn_method='cuda' gets the caller's float32 array itself (validated, not copied); the
    other methods get the float64 copy the reference makes; NaN is refused either way. The
    k-NN and the backend are stand-ins here, so no device is needed."""
    from scipy.sparse import csr_matrix
    import tsne_h2pack.manifold as M
    import tsne_h2pack._knn_methods as K
    real = M.get_backend()
    seen = {}

    class FakeKNN:
        def compute(self, X, k, **kw):
            seen["knn_X"] = X
            n = X.shape[0]
            idx = (np.arange(n)[:, None] + np.arange(1, k + 1)[None, :]) % n
            return csr_matrix((np.ones(n * k), idx.ravel(), np.arange(0, (n + 1) * k, k)), shape=(n, n))

    class FakeBackend:
        backend_type = "stand-in"
        create_default_params = staticmethod(real.create_default_params)

        def fit_transform_with_knn_distances(self, X, G, c, params, init_Y=None):
            seen["X"] = X
            return np.zeros((X.shape[0], c)), {"kl_divergence": 0.0, "n_iter": 1}

    monkeypatch.setattr(K, "get_knn_method", lambda name: FakeKNN())
    monkeypatch.setattr(M, "get_backend", lambda: FakeBackend())
    X = np.random.default_rng(0).standard_normal((100, 5)).astype(np.float32)
    TSNE(knn_method="cuda", perplexity=5, init="random").fit_transform(X)
    assert seen["knn_X"] is X and seen["X"] is X
    TSNE(knn_method="exact", perplexity=5, init="random").fit_transform(X)
    assert seen["knn_X"].dtype == np.float64
    np.testing.assert_array_equal(seen["knn_X"], X.astype(np.float64))
    Xn = X.copy()
    Xn[3, 1] = np.nan
    with pytest.raises(ValueError):
        TSNE(knn_method="cuda", perplexity=5, init="random").fit_transform(Xn)
