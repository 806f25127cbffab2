"""Edge cases of the device engine against the oracle: malformed P rejected on the host,
ragged P (isolated points, a hub row), user leaf sizes on both sides of the 2D basis kernels'
128-row limit, and a block of coincident points (a leaf at the key depth holding more than
leaf_size points).

Tolerances as in test_gpu_engine.py: tree permutation, node table and lists bit-exact;
H2 force within h2_tol of the FP64 exact force; attractive force rel 1e-5; KL within 0.5%
after 29 iterations of the full schedule.
"""
import ctypes

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, problem, rel, rel2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mid():
    return problem(5000, seed=1, n_clusters=12, dim=20)


def _evolved(P, n_iter, seed):
    Y0 = O.init_embedding(P.shape[0], 2, seed)
    return O.run(P, Y0, n_iter=n_iter)[0].astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("bad", [-1, "n"])
def test_out_of_range_column_is_rejected(bad):
    """A column index outside [0, n) makes tsne_init_with_P return NULL (checked on the host
    while P is staged, before the device reads any index)."""
    X, G, P, _ = problem(1000, seed=0)
    P = P.tocsr().copy()
    P.indices[P.indptr[17] + 1] = P.shape[0] if bad == "n" else bad
    with pytest.raises(RuntimeError):
        Engine(P, O.init_embedding(P.shape[0], 2, 1), n_iter=1)


def _ragged(P, seed=0):
    """P with 10 isolated points (no entries in their rows or columns) and one hub point tied
    to 3000 others, symmetric and normalised to sum 1."""
    rng = np.random.default_rng(seed)
    n = P.shape[0]
    A = P.tocoo()
    iso = np.arange(1, 11)
    keep = ~(np.isin(A.row, iso) | np.isin(A.col, iso))
    rows, cols, vals = A.row[keep], A.col[keep], A.data[keep]
    others = rng.choice(np.arange(11, n), 3000, replace=False)
    w = rng.uniform(0.5, 1.5, others.size) * vals.mean()
    rows = np.concatenate([rows, np.zeros(others.size, int), others])
    cols = np.concatenate([cols, others, np.zeros(others.size, int)])
    vals = np.concatenate([vals, w, w])
    Q = csr_matrix((vals, (rows, cols)), shape=(n, n))
    Q.sum_duplicates()
    Q.sort_indices()
    Q.data /= Q.data.sum()
    return Q


def test_ragged_rows(mid, monkeypatch):
    """Empty rows and a 3000-entry row through the attractive pass (C ABI) and the full
    schedule with renumbering at iterations 5 and 12 (rows of every length gathered)."""
    from tsne_h2pack._backend import scipy_csr_to_c_sparse_matrix
    X, G, P, _ = mid
    Q = _ragged(P)
    lens = np.diff(Q.indptr)
    assert lens[1:11].max() == 0 and lens[0] >= 3000
    Y = _evolved(Q, 50, 3)
    eng = Engine(Q, Y, n_iter=1)
    grad = np.zeros_like(Y)
    Pc = scipy_csr_to_c_sparse_matrix(Q, eng.lib)
    eng.lib.compute_attractive_forces(ctypes.cast(Pc, ctypes.c_void_p), np.ascontiguousarray(Y), 2, Y.shape[1],
                                      12.0, grad, 1)
    eng.lib.sparse_matrix_destroy(Pc)
    eng.close()
    assert rel(grad, O.attractive(Q, Y, 12.0)) < 1e-5
    monkeypatch.setenv("TSNE_REORDER_ITERS", "5,12")
    Y0 = O.init_embedding(Q.shape[0], 2, 4)
    eng = Engine(Q, Y0, n_iter=29)
    eng.run_all()
    kld = eng.kl()
    eng.close()
    Yo, klo = O.run(Q, Y0, n_iter=29)
    print("ragged P: KL device", kld, "oracle", klo)
    assert abs(kld - klo) < 5e-3 * abs(klo)


def _check_h2(P, Y, leaf):
    eng = Engine(P, Y, n_iter=1, h2_leaf_size=leaf)
    assert eng.rebuild() == 0
    dev = eng.h2()
    h = O.H2(Y, leaf_size=leaf, tol=1e-2)
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
    sizes = (on["end"] - on["start"])[on["is_leaf"] == 1]
    F, Z = eng.repulsive(Y)
    eng.close()
    s, v = O.exact_sv(Y)
    Ze, Fe = O.z_force(Y, s, v)
    print(f"leaf {leaf}: largest leaf {sizes.max()}, force rel {rel2(F, Fe):.3e}, Z rel {abs(Z - Ze) / Ze:.3e}")
    assert rel2(F, Fe) <= 1e-2
    assert abs(Z - Ze) <= 1e-2 * Ze
    return sizes.max()


@pytest.mark.parametrize("leaf", [40, 160])
def test_leaf_size_parameter(mid, leaf):
    """h2_leaf_size 40 (deeper tree, 2D shared-memory bases) and 160 (leaves above 128 rows:
    the general basis kernel in 2D)."""
    X, G, P, _ = mid
    Y = _evolved(P, 300, 2)
    biggest = _check_h2(P, Y, leaf)
    assert biggest <= leaf


def test_coincident_points(mid):
    """150 points at one position: the tree splits down to the key depth, where one leaf holds
    all of them (more than leaf_size 100)."""
    X, G, P, _ = mid
    Y = _evolved(P, 300, 2)
    idx = np.random.default_rng(5).choice(P.shape[0], 150, replace=False)
    Y[:, idx] = Y[:, idx[:1]]
    biggest = _check_h2(P, Y, 100)
    assert biggest >= 150


def test_dependency_wait_timeout_is_reported(mid):
    """The failure path of the bounded waits in the dependency-ordered H2 launches: one wait,
    limited to 1000 polls, on a node flag that nothing publishes gives up and records the
    failure; the workspace's next run reports it (-1) instead of using the matrix, and a new
    workspace in the same process still runs (the device context is intact)."""
    X, G, P, _ = mid
    Y0 = O.init_embedding(P.shape[0], 2, 4)
    eng = Engine(P, Y0, n_iter=40)
    lib = eng.lib
    lib.tsne_h2_probe_dependency_timeout.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.tsne_h2_probe_dependency_timeout.restype = ctypes.c_int
    eng.run(0, 5)
    h = lib.tsne_get_h2_matrix(eng.ws)
    assert h
    assert lib.tsne_h2_probe_dependency_timeout(h, 0) == -1          # out of range: nothing launched
    assert lib.tsne_h2_probe_dependency_timeout(h, 1000) == 1
    with pytest.raises(RuntimeError):
        eng.run(5, 10)
    eng.close()
    eng = Engine(P, Y0, n_iter=29)
    eng.run_all()
    _, klo = O.run(P, Y0, n_iter=29)
    assert abs(eng.kl() - klo) < 5e-3 * abs(klo)
    eng.close()
