"""Parity of the device engine (through its C ABI) with the oracle and the reference.

Tolerances (FP32 device state against FP64 oracles; t-SNE amplifies a rounding difference
by roughly 2x per iteration, so trajectory comparisons stop after a few tens of
iterations):
  - exact path vs the reference's own build: max rel 1e-5 after 1 iteration, 1e-4 after 5;
    KL within 0.1% after 10 iterations and 1% after 20
  - perplexity calibration vs the oracle: rtol 1e-10
  - H2 tree permutation, node table and near/far lists vs the oracle: bit-exact
  - H2 repulsive force vs the FP64 exact force: rel 2-norm <= h2_tol
  - fused force product vs the general-column product of the same H2 matrix: rel 2e-5
  - full schedule vs the oracle: embedding rel 1e-2 after 3 iterations, KL 0.5% after 29
  - attractive force vs the FP64 oracle: rel 1e-5
  - 1000-iteration run: KL within 1% of the oracle's run, 30-NN preservation within 0.5 points
"""
import ctypes

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, knn_preservation, problem, rel, rel2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return problem(1000, seed=0)


@pytest.fixture(scope="module")
def mid():
    return problem(5000, seed=1, n_clusters=12, dim=20)


def test_exact_path_matches_reference(small):
    """N < 2000 runs the exact O(N^2) repulsion every iteration, as the reference does. The
    device state is FP32: its rounding grows ~2x per iteration like any t-SNE perturbation
    (the FP64 oracle and the reference's own build drift apart the same way), so the
    embeddings are compared after 5 iterations and the KL after 10 and 20."""
    X, G, P, _ = small
    Y0 = O.init_embedding(P.shape[0], 2, 11)
    ref = (lambda it: O.ref_run(P, Y0, it, learning_rate=200.0)) if O.ref_available() else \
        (lambda it: O.run(P, Y0, n_iter=it, learning_rate=200.0, use_h2=False))
    for n_iter, tol in ((1, 1e-5), (5, 1e-4)):
        eng = Engine(P, Y0, n_iter=n_iter, learning_rate=200.0)
        eng.run_all()
        assert rel(eng.embedding(), ref(n_iter)[0]) < tol, n_iter
        eng.close()
    for n_iter, tol in ((10, 1e-3), (20, 1e-2)):
        eng = Engine(P, Y0, n_iter=n_iter, learning_rate=200.0)
        eng.run_all()
        Yr, klr = ref(n_iter)
        assert abs(eng.kl() - klr) < tol * abs(klr), n_iter


def test_exact_method_matches_oracle(mid):
    """method='exact' (h2_rebuild_freq = 999999) at N >= 2000."""
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 2, 5)
    eng = Engine(P, Y0, n_iter=5, exact=True)
    eng.run_all()
    Yo, _ = O.run(P, Y0, n_iter=5, use_h2=False)
    assert rel(eng.embedding(), Yo) < 1e-4
    eng = Engine(P, Y0, n_iter=15, exact=True)
    eng.run_all()
    Yo, klo = O.run(P, Y0, n_iter=15, use_h2=False)
    assert abs(eng.kl() - klo) < 1e-3 * abs(klo)


def test_conditional_P_matches_oracle(small):
    from tsne_h2pack._backend import get_backend
    X, G, P, _ = small
    Pc = get_backend().conditional_P(G, 30.0)
    ref = O.conditional_P(G.data, G.indptr, 30.0)
    np.testing.assert_allclose(Pc.data, ref, rtol=1e-10, atol=1e-300)


@pytest.mark.parametrize("scale", [1e-3, 1.0, 1e3, 1e6])
def test_calibration_known_answers(scale):
    """Rows sum to 1 and hit perplexity 30; scale invariant (the reference's
    tests/test_perplexity_calibration.py:18-59 on the same fixture)."""
    from tsne_h2pack._backend import get_backend
    rng = np.random.default_rng(0)
    d = np.sort(rng.uniform(1.0, 3.0, size=(200, 90)), axis=1)
    n, k = d.shape
    G = csr_matrix((d.ravel() * scale, np.tile(np.arange(k), n), np.arange(0, (n + 1) * k, k)), shape=(n, 200))
    be = get_backend()
    Pc = be.conditional_P(G, 30.0).toarray()[:, :k]
    base = be.conditional_P(csr_matrix((d.ravel(), G.indices, G.indptr), shape=(n, 200)), 30.0).toarray()[:, :k]
    np.testing.assert_allclose(Pc.sum(axis=1), 1.0, rtol=1e-10)
    H = -np.sum(np.where(Pc > 0, Pc * np.log2(np.maximum(Pc, 1e-300)), 0.0), axis=1)
    np.testing.assert_allclose(2.0 ** H, 30.0, rtol=1e-3)
    np.testing.assert_allclose(Pc, base, rtol=1e-3, atol=1e-9)


def _evolved(P, n_iter, seed):
    Y0 = O.init_embedding(P.shape[0], 2, seed)
    Y, _ = O.run(P, Y0, n_iter=n_iter)
    return Y


@pytest.mark.parametrize("n_iter", [20, 300])
def test_tree_and_lists_bit_exact(mid, n_iter):
    X, G, P, _ = mid
    Y = _evolved(P, n_iter, 2).astype(np.float32).astype(np.float64)
    eng = Engine(P, Y, n_iter=1)
    assert eng.rebuild() == 0
    dev = eng.h2()
    assert dev is not None
    h = O.H2(Y, leaf_size=100, tol=1e-2)
    corner, radius = h.root()
    assert radius == dev["radius"]
    np.testing.assert_array_equal(corner, dev["corner"])
    np.testing.assert_array_equal(h.perm(), dev["perm"])
    assert h.n_node == dev["n_node"] and h.max_level == dev["max_level"]
    on = h.nodes()
    for k in on:
        np.testing.assert_array_equal(on[k], dev["nodes"][k], err_msg=k)
    fp, fi, np_, ni = h.lists()
    np.testing.assert_array_equal(fp, dev["far_ptr"])
    np.testing.assert_array_equal(fi, dev["far_idx"])
    np.testing.assert_array_equal(np_, dev["near_ptr"])
    np.testing.assert_array_equal(ni, dev["near_idx"])


@pytest.mark.parametrize("n_iter", [20, 100, 300, 1000])
def test_h2_force_within_tolerance(mid, n_iter):
    X, G, P, _ = mid
    Y = _evolved(P, n_iter, 2).astype(np.float32).astype(np.float64)
    eng = Engine(P, Y, n_iter=1)
    assert eng.rebuild() == 0
    F, Z = eng.repulsive(Y)
    s, v = O.exact_sv(Y)
    Ze, Fe = O.z_force(Y, s, v)
    err = rel2(F, Fe)
    print(f"iter {n_iter}: force rel {err:.3e}, Z rel {abs(Z - Ze) / Ze:.3e}, ranks max {eng.h2()['ranks'].max()}")
    assert err <= 1e-2
    assert abs(Z - Ze) <= 1e-2 * Ze


@pytest.mark.parametrize("n_iter", [20, 300])
def test_force_path_matches_general_product(mid, n_iter):
    """The fused force product of the iteration ([1 | x y] columns, two target points per
    thread) against the general-column product of the same H2 matrix (tsne_h2_matmul), from
    which s, v, Z and the force follow by the reference's identities: both FP32, so they agree
    to rounding (rel 2e-5)."""
    X, G, P, _ = mid
    Y = _evolved(P, n_iter, 2).astype(np.float32).astype(np.float64)
    eng = Engine(P, Y, n_iter=1)
    assert eng.rebuild() == 0
    F, Z = eng.repulsive(Y)
    W = eng.matmul([np.ones(Y.shape[1]), Y[0], Y[1]])
    eng.close()
    Zg, Fg = O.z_force(Y, W[0] - 1.0, W[1:] - Y)
    print(f"iter {n_iter}: force rel {rel2(F, Fg):.3e}, Z rel {abs(Z - Zg) / Zg:.3e}")
    assert rel2(F, Fg) < 2e-5
    assert abs(Z - Zg) < 2e-5 * Zg


@pytest.fixture(scope="module")
def evolved3d(mid):
    """3D embeddings of the mid problem after 20 and 150 iterations of the oracle's run."""
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 3, 6)
    return P, {it: O.run(P, Y0, n_iter=it)[0].astype(np.float32).astype(np.float64) for it in (20, 150)}


@pytest.mark.parametrize("n_iter", [20, 150])
def test_h2_3d_tree_lists_and_force(evolved3d, n_iter):
    """3D: tree permutation, node table and lists bit-exact against the oracle; the H2 force
    (shared-memory ID with grouped rows) within h2_tol of the exact FP64 force."""
    P, Ys = evolved3d
    Y = Ys[n_iter]
    eng = Engine(P, Y, n_iter=1)
    assert eng.rebuild() == 0
    dev = eng.h2()
    h = O.H2(Y, leaf_size=100, tol=1e-2)
    np.testing.assert_array_equal(h.perm(), dev["perm"])
    on = h.nodes()
    for k in on:
        np.testing.assert_array_equal(on[k], dev["nodes"][k], err_msg=k)
    fp, fi, np_, ni = h.lists()
    np.testing.assert_array_equal(fi, dev["far_idx"])
    np.testing.assert_array_equal(ni, dev["near_idx"])
    F, Z = eng.repulsive(Y)
    eng.close()
    s, v = O.exact_sv(Y)
    Ze, Fe = O.z_force(Y, s, v)
    print(f"3D iter {n_iter}: force rel {rel2(F, Fe):.3e}, Z rel {abs(Z - Ze) / Ze:.3e}")
    assert rel2(F, Fe) <= 1e-2
    assert abs(Z - Ze) <= 1e-2 * Ze


def test_attractive_matches_oracle(mid):
    from tsne_h2pack._backend import scipy_csr_to_c_sparse_matrix
    X, G, P, _ = mid
    Y = _evolved(P, 50, 3)
    eng = Engine(P, Y, n_iter=1)
    grad = np.zeros_like(Y)
    Pc = scipy_csr_to_c_sparse_matrix(P, eng.lib)
    eng.lib.compute_attractive_forces(ctypes.cast(Pc, ctypes.c_void_p), np.ascontiguousarray(Y), 2, Y.shape[1],
                                      12.0, grad, 1)
    eng.lib.sparse_matrix_destroy(Pc)
    ref = O.attractive(P, Y, 12.0)
    assert rel(grad, ref) < 1e-5


def test_short_trajectory_matches_oracle(mid):
    """Full schedule (H2 rebuild every iteration below 20). The device skeletons differ from
    the FP64 oracle's at the ID tolerance, a perturbation that t-SNE amplifies, so the
    embeddings are compared after 3 iterations (rel 1e-2) and the KL after 29 (0.5%)."""
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 2, 4)
    eng = Engine(P, Y0, n_iter=3)
    eng.run_all()
    r = rel(eng.embedding(), O.run(P, Y0, n_iter=3)[0])
    eng.close()
    eng = Engine(P, Y0, n_iter=29)
    eng.run_all()
    Yo, klo = O.run(P, Y0, n_iter=29)
    print("3-iteration rel", r, "KL", eng.kl(), klo)
    assert r < 1e-2
    assert abs(eng.kl() - klo) < 5e-3 * abs(klo)


def test_renumbering_is_transparent(mid, monkeypatch):
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 2, 8)
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("TSNE_REORDER", flag)
        eng = Engine(P, Y0, n_iter=34)
        eng.run_all()
        out[flag] = eng.embedding()
        eng.close()
    assert rel(out["1"], out["0"]) < 1e-3


def test_deterministic(mid):
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 2, 9)
    a = Engine(P, Y0, n_iter=40); a.run_all()
    b = Engine(P, Y0, n_iter=40); b.run_all()
    np.testing.assert_array_equal(a.embedding(), b.embedding())


def test_full_run_quality():
    """C1-shaped run (10K x 50, 10 clusters, k = 90, perplexity 30, 1000 iterations): KL within
    1% of the oracle's run and 30-NN preservation within 0.5 points."""
    X, G, P, _ = problem(10000, seed=0)
    Y0 = O.init_embedding(P.shape[0], 2, 0)
    eng = Engine(P, Y0, n_iter=1000)
    eng.run_all()
    Yd, kld = eng.embedding(), eng.kl()
    Yo, klo = O.run(P, Y0, n_iter=1000)
    pd, po = knn_preservation(X, Yd.T), knn_preservation(X, Yo.T)
    print(f"KL device {kld:.5f} oracle {klo:.5f}; 30-NN device {pd:.4f} oracle {po:.4f}")
    assert abs(kld - klo) <= 0.01 * klo
    assert abs(pd - po) <= 0.005


def test_nonfinite_embedding_is_rejected(mid):
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 2, 1)
    Y0[0, 7] = np.nan
    with pytest.raises(RuntimeError):
        Engine(P, Y0, n_iter=5)


def test_python_api_precomputed_matches_euclidean():
    """The precomputed-graph path equals the feature path (reference test_tsne.py:765-811)."""
    from tsne_h2pack import TSNE
    X, G, P, _ = problem(3000, seed=5, dim=20)
    kw = dict(n_components=2, perplexity=30, max_iter=40, init="random", random_state=3, knn_method="exact")
    Ya = TSNE(**kw).fit_transform(X)
    Yb = TSNE(metric="precomputed", **kw).fit_transform(G)
    np.testing.assert_array_equal(Ya, Yb)
