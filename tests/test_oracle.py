"""The CPU oracle, pinned against the reference's own sources (built under oracle/_ref) and
the reference's known-answer tests. CPU only."""
import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import problem, rel, rel2

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")


@pytest.fixture(scope="module")
def small():
    return problem(1000, seed=0)


@needs_ref
def test_init_embedding_equals_reference():
    """Same C library generator (srand / Box-Muller) as the reference; the reference build
    uses -ffast-math, so the transcendental rounding may differ in the last bits."""
    for n, d, seed in ((1000, 2, 42), (777, 3, 0), (5, 2, 123456)):
        np.testing.assert_allclose(O.init_embedding(n, d, seed), O.ref_init_embedding(n, d, seed), rtol=1e-11,
                                   atol=0)


def test_engine_init_embedding_equals_oracle():
    """The engine's initialize_embedding is host code with its own copy of the C library's
    rand() sequence: bit-identical to the oracle's, which calls srand/rand (seeds with the top
    bit set included, an odd number of values, 3D)."""
    import ctypes
    from tsne_h2pack._backend import get_backend
    lib = get_backend()._lib
    lib.initialize_embedding.argtypes = [np.ctypeslib.ndpointer(np.float64), ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_uint]
    for n, d, seed in ((1000, 2, 42), (777, 3, 0), (100001, 2, 3000000000), (300000, 3, 2**32 - 1), (7, 3, 1),
                       (64, 2, 2**31)):
        Y = np.zeros((d, n))
        lib.initialize_embedding(Y, n, d, 0, None, seed)
        np.testing.assert_array_equal(Y, O.init_embedding(n, d, seed))


@needs_ref
def test_conditional_P_equals_reference(small):
    X, G, P, _ = small
    a = O.conditional_P(G.data, G.indptr, 30.0)
    b = O.ref_conditional_P(G.data, G.indices, G.indptr, 30.0)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)


@needs_ref
@pytest.mark.parametrize("n_iter", [1, 10, 20])
def test_exact_trajectory_equals_reference(small, n_iter):
    """The whole loop on the exact path (attractive, exact repulsion, Z identity, update,
    centring, KL) against the reference's tsne_run: FP64 vs FP64 (the reference is built with
    -ffast-math), so only rounding separates them."""
    X, G, P, _ = small
    Y0 = O.init_embedding(P.shape[0], 2, 11)
    Yr, klr = O.ref_run(P, Y0, n_iter, learning_rate=200.0)
    Yo, klo = O.run(P, Y0, n_iter=n_iter, learning_rate=200.0, use_h2=False)
    assert rel(Yo, Yr) < 1e-9
    assert abs(klo - klr) < 1e-9 * abs(klr)


@pytest.mark.parametrize("scale", [1e-3, 1.0, 1e3, 1e6])
def test_calibration_known_answers(scale):
    """Reference tests/test_perplexity_calibration.py:18-59 on the oracle: rows sum to 1, hit
    perplexity 30, scale invariant."""
    rng = np.random.default_rng(0)
    d = np.sort(rng.uniform(1.0, 3.0, size=(200, 90)), axis=1)
    ptr = np.arange(0, 201 * 90, 90)
    P = O.conditional_P((d * scale).ravel(), ptr, 30.0).reshape(200, 90)
    base = O.conditional_P(d.ravel(), ptr, 30.0).reshape(200, 90)
    np.testing.assert_allclose(P.sum(axis=1), 1.0, rtol=1e-10)
    H = -np.sum(np.where(P > 0, P * np.log2(np.maximum(P, 1e-300)), 0.0), axis=1)
    np.testing.assert_allclose(2.0 ** H, 30.0, rtol=1e-3)
    np.testing.assert_allclose(P, base, rtol=1e-3, atol=1e-9)


def test_kl_matches_sklearn():
    """The exact KL divergence against scikit-learn's implementation (dense P, dof 1)."""
    from sklearn.manifold._t_sne import _kl_divergence
    X, G, P, _ = problem(300, seed=4, k=60, perplexity=15.0, dim=10, n_clusters=3)
    Y = O.init_embedding(300, 2, 3) * 1e3
    s, v = O.exact_sv(Y)
    Z, F = O.z_force(Y, s, v)
    kl = O.kl(P, Y, 1.0, Z)
    from scipy.spatial.distance import squareform
    Pd = P.toarray()
    kl_sk, grad_sk = _kl_divergence(Y.T.ravel().copy(), squareform(Pd, checks=False), 1.0, 300, 2)
    assert abs(kl - kl_sk) < 1e-10 * abs(kl_sk)
    # sklearn's gradient = 4 (attractive - repulsive) with the exact Z
    attr = O.attractive(P, Y, 1.0)
    g = (attr - F).T.ravel()
    assert rel2(g, grad_sk) < 1e-9


@pytest.fixture(scope="module")
def evolved():
    X, G, P, _ = problem(3000, seed=1, n_clusters=12, dim=20)
    out = {}
    for it in (20, 300):
        out[it] = O.run(P, O.init_embedding(3000, 2, 2), n_iter=it)[0].astype(np.float32).astype(np.float64)
    return out


@pytest.mark.parametrize("it", [20, 300])
def test_h2_lists_cover_every_pair_once(evolved, it):
    """Every ordered pair (i, j) lies in exactly one far or near block of the target's lists."""
    Y = evolved[it]
    h = O.H2(Y, leaf_size=50, tol=1e-2)
    nd = h.nodes()
    perm = h.perm()
    pos = np.empty_like(perm); pos[perm] = np.arange(len(perm))
    fp, fi, np_, ni = h.lists()
    n = Y.shape[1]
    cover = np.zeros((n, n), dtype=np.int32)
    for ptr, idx in ((fp, fi), (np_, ni)):
        for t in range(h.n_node):
            for s in idx[ptr[t]:ptr[t + 1]]:
                cover[nd["start"][t]:nd["end"][t], nd["start"][s]:nd["end"][s]] += 1
    assert cover.min() == 1 and cover.max() == 1


@pytest.mark.parametrize("name", ["3D gaussian", "3D clusters", "2D coincident block"])
def test_h2_lists_cover_every_pair_once_more_shapes(name):
    """The same cover property in 3D and with a block of coincident points (a leaf at the key
    depth holding more than leaf_size points)."""
    rng = np.random.default_rng(3)
    if name == "3D gaussian":
        Y, leaf = rng.normal(size=(3, 2500)), 40
    elif name == "3D clusters":
        Y, leaf = rng.normal(size=(3, 2500)) * 1e-2 + rng.integers(0, 4, size=(3, 2500)), 40
    else:
        Y, leaf = rng.normal(size=(2, 2500)), 40
        Y[:, 100:260] = 0.5
    h = O.H2(Y, leaf_size=leaf, tol=1e-2)
    nd = h.nodes()
    fp, fi, np_, ni = h.lists()
    n = Y.shape[1]
    cover = np.zeros((n, n), dtype=np.int32)
    for ptr, idx in ((fp, fi), (np_, ni)):
        for t in range(h.n_node):
            for s in idx[ptr[t]:ptr[t + 1]]:
                cover[nd["start"][t]:nd["end"][t], nd["start"][s]:nd["end"][s]] += 1
    assert cover.min() == 1 and cover.max() == 1


@pytest.mark.parametrize("it", [20, 300])
def test_h2_lists_symmetric(evolved, it):
    h = O.H2(evolved[it], leaf_size=50, tol=1e-2)
    fp, fi, np_, ni = h.lists()
    for ptr, idx in ((fp, fi), (np_, ni)):
        pairs = {(t, s) for t in range(h.n_node) for s in idx[ptr[t]:ptr[t + 1]]}
        assert all((s, t) in pairs for t, s in pairs)


@pytest.mark.parametrize("it", [20, 300])
def test_h2_product_within_tolerance(evolved, it):
    """Oracle H2 force vs the exact FP64 force: within h2_tol."""
    Y = evolved[it]
    h = O.H2(Y, leaf_size=100, tol=1e-2)
    s, v = h.product()
    se, ve = O.exact_sv(Y)
    Z, F = O.z_force(Y, s, v)
    Ze, Fe = O.z_force(Y, se, ve)
    assert rel2(F, Fe) < 1e-2
    assert abs(Z - Ze) < 1e-2 * Ze


@needs_ref
@pytest.mark.parametrize("d,it,leaf", [(2, 20, 100), (2, 300, 50), (3, 150, 100)])
def test_h2_force_equals_reference_code_on_the_same_matrix(d, it, leaf):
    """The reference's own compute_repulsive_forces_h2pack (its fused product
    tsne_h2_matmul.c:225-452, diagonal removal, Z identity and force, tsne_h2pack.c:389-630),
    compiled from its sources and handed the oracle's H2 matrix (tree, reduced admissible and
    inadmissible pair lists, bases, skeletons), gives the oracle's product, Z and force to
    rounding: the oracle's far/near traversal, mixed-level pairs, upward and downward passes
    and force assembly are the reference's."""
    X, G, P, _ = problem(3000, seed=1, n_clusters=12, dim=20)
    Y = O.run(P, O.init_embedding(3000, d, 2), n_iter=it)[0]
    h = O.H2(Y, leaf_size=leaf, tol=1e-2)
    Fr, Zr = O.ref_h2_repulsion(h)
    s, v = h.product()
    Zo, Fo = O.z_force(Y, s, v)
    assert abs(Zr - Zo) <= 1e-11 * Zo
    assert rel2(Fr, Fo) <= 1e-11


@needs_ref
@pytest.mark.parametrize("d,n_iter,tol_y,tol_kl", [(2, 25, 1e-9, 1e-11), (2, 40, 1e-4, 1e-8), (3, 30, 1e-5, 1e-9),
                                                   (3, 35, 1e-4, 1e-7)])
def test_reference_loop_on_oracle_matrices_equals_oracle_run(d, n_iter, tol_y, tol_kl):
    """The reference's own tsne_run on its H2 path (tsne_h2pack.c:1652-2102: rebuild every
    iteration below 20 and every 10 after, force and Z reuse between rebuilds, renumbering at
    the first rebuild >= 30, its update, centring and KL), with every H2 matrix built by the
    oracle behind the H2Pack interface (ref_shim/h2_assemble.c) and its FP64 attractive pass,
    follows the oracle's own run: to rounding through 25 iterations, and after the
    renumbering at iteration 30 (40 iterations) to the ~2x-per-iteration growth of rounding
    differences that t-SNE shows, KL to 1e-8."""
    X, G, P, _ = problem(5000, seed=1, n_clusters=12, dim=20)
    Y0 = O.init_embedding(P.shape[0], d, 4)
    Yr, klr = O.ref_run(P, Y0, n_iter, h2=True, attr_generic=True, nthreads=4)
    Yo, klo = O.run(P, Y0, n_iter=n_iter)
    assert rel(Yr, Yo) < tol_y
    assert abs(klr - klo) <= tol_kl * abs(klo)


def _zipf_cloud(n, d, spread, seed):
    """n points in d dimensions: 100 Gaussian clusters of Zipf(1.1) sizes (a stand-in for a
    converged embedding of the benchmark's mixture), rounded to float32."""
    rng = np.random.default_rng(seed)
    w = np.arange(1, 101) ** -1.1
    cnt = rng.multinomial(n, w / w.sum())
    cen = rng.normal(0, spread, (100, d))
    sd = rng.uniform(1, 4, (100, d))
    lab = np.repeat(np.arange(100), cnt)
    Y = (cen[lab] + sd[lab] * rng.standard_normal((n, d))).T
    return np.ascontiguousarray(Y).astype(np.float32).astype(np.float64), rng


@pytest.mark.parametrize("n,d,tol", [(1_000_000, 2, 1e-2), (500_000, 3, 3e-2)])
def test_h2_accuracy_at_full_size(n, d, tol):
    """At the benchmark sizes (1M points in 2D with h2_tol 1e-2; 500K in 3D with 3e-2), the H2
    sums of 400 random points against their exact FP64 sums over all points: s and v within
    tol / 5, the force numerator y s - v within tol. (Exact sums for every point are out of
    reach at this size; the sampled rows check the same property.)"""
    Y, rng = _zipf_cloud(n, d, 40.0 if d == 2 else 25.0, 7 + d)
    h = O.H2(Y, leaf_size=100, tol=tol)
    s, v = h.product()
    rows = np.sort(rng.choice(n, 400, replace=False))
    se, ve = O.exact_rows(Y, rows)
    assert rel2(s[rows], se) < tol / 5 and rel2(v[:, rows], ve) < tol / 5
    assert rel2(Y[:, rows] * s[rows] - v[:, rows], Y[:, rows] * se - ve) < tol


def test_exact_rows_equal_exact_sums():
    Y = O.init_embedding(3000, 3, 5) * 1e3
    rows = np.array([0, 17, 1500, 2999], dtype=np.int32)
    s, v = O.exact_sv(Y)
    sr, vr = O.exact_rows(Y, rows)
    np.testing.assert_array_equal(sr, s[rows])
    np.testing.assert_array_equal(vr, v[:, rows])


def test_tree_is_a_partition(evolved):
    h = O.H2(evolved[300], leaf_size=40, tol=1e-2)
    nd = h.nodes()
    leaf = nd["is_leaf"].astype(bool)
    cnt = np.zeros(h.n, dtype=int)
    for s, e in zip(nd["start"][leaf], nd["end"][leaf]):
        cnt[s:e] += 1
    assert (cnt == 1).all()
    assert np.array_equal(np.sort(h.perm()), np.arange(h.n))
    keys = h.keys()
    assert (np.diff(keys.astype(np.float64)) >= 0).all()
    # internal nodes hold more than leaf_size points, leaves at most (below the depth limit)
    sizes = nd["end"] - nd["start"]
    assert (sizes[~leaf] > 40).all() and (sizes[leaf] <= 40).all()


def test_shallow_tree_reports_status():
    Y = O.init_embedding(150, 2, 1)
    h = O.H2(Y, leaf_size=100, tol=1e-2)
    assert h.status == 1
