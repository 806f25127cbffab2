"""P built on the device (tsne_joint_P_from_knn_distances, tsne_init_with_knn_distances)
against the reference's host computation (device calibration, then scipy's P + P^T and the
division by the total, reference tsne_h2pack/_backend.py:709-718):

  - structure (row pointers, columns) identical; values equal to rel 1e-12 (they differ only
    by the rounding of the normalising total); the unnormalised sums equal bit for bit;
  - ragged graphs: isolated rows, rows of one neighbour, asymmetric neighbourhoods, and
    entries whose probability underflows to zero (dropped on both sides);
  - malformed graphs rejected before the device reads an index: decreasing row pointers,
    unsorted rows, self entries, columns outside [0, n);
  - a workspace made from the graph (P never on the host) runs as one made from the host P:
    embedding after 60 iterations within 1e-6, KL within 1e-6 (single-precision P entries are
    the same floats unless a value sits on a rounding boundary).
"""
import ctypes

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, problem, rel

pytestmark = pytest.mark.gpu


def _be():
    from tsne_h2pack._backend import get_backend
    return get_backend()


def _compare(G, perp):
    be = _be()
    Ph = be.joint_P(G, perp)
    Pd = be.joint_P_device(G, perp)
    Ph.sort_indices()
    np.testing.assert_array_equal(Ph.indptr, Pd.indptr)
    np.testing.assert_array_equal(Ph.indices, Pd.indices)
    np.testing.assert_allclose(Pd.data, Ph.data, rtol=1e-12, atol=0)
    # the same sums before normalisation: the ratio of the two matrices is one number
    ratio = Pd.data / Ph.data
    assert np.ptp(ratio) <= 2e-15 * ratio.mean()
    return Ph, Pd


@pytest.mark.parametrize("n,k,perp", [(3000, 45, 15.0), (20000, 90, 30.0)])
def test_device_P_matches_host_P(n, k, perp):
    X, G, P, _ = problem(n, seed=3, k=k, perplexity=perp, dim=20)
    _compare(G.tocsr(), perp)


def test_device_P_ragged_graph():
    rng = np.random.default_rng(1)
    n = 2500
    rows, cols, vals = [], [], []
    iso = np.arange(0, n, 97)                               # isolated rows: no entries, nobody's neighbour
    pool = np.setdiff1d(np.arange(n), iso)
    for i in range(n):
        if i % 97 == 0:
            continue
        k = 1 if i % 13 == 0 else int(rng.integers(5, 60))
        nb = np.sort(rng.choice(pool[pool != i], size=k, replace=False))
        d = np.sort(rng.uniform(0.5, 3.0, size=k))
        if i % 29 == 0:
            d[-1] = 1e4                                     # far neighbour: its probability underflows
        rows += [i] * k; cols += nb.tolist(); vals += d[np.argsort(np.argsort(nb))].tolist()
    G = csr_matrix((vals, (rows, cols)), shape=(n, n))
    G.sort_indices()
    Ph, Pd = _compare(G, 10.0)
    assert (np.diff(Pd.indptr) == 0).sum() >= 1


def _call(G_data, G_ind, G_ptr, n):
    be = _be()
    d = np.ascontiguousarray(G_data, dtype=np.float64)
    i = np.ascontiguousarray(G_ind, dtype=np.int32)
    p = np.ascontiguousarray(G_ptr, dtype=np.int32)
    return be._lib.tsne_joint_P_from_knn_distances(d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                   i.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                   p.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, len(d),
                                                   ctypes.c_double(5.0))


def test_malformed_graphs_are_rejected():
    n = 50
    ptr = np.arange(0, 3 * n + 1, 3)
    ind = np.array([[(i + 1) % n, (i + 2) % n, (i + 3) % n] for i in range(n)])
    ind.sort(axis=1)
    d = np.ones(3 * n)
    ok = _call(d, ind.ravel(), ptr, n)
    assert ok
    _be()._lib.sparse_matrix_destroy(ok)
    bad_ptr = ptr.copy(); bad_ptr[10] = bad_ptr[11] + 1
    assert not _call(d, ind.ravel(), bad_ptr, n)               # decreasing row pointers (host check)
    big_ptr = ptr.copy(); big_ptr[-1] += 5
    assert not _call(d, ind.ravel(), big_ptr, n)               # last pointer != nnz
    uns = ind.copy(); uns[4] = uns[4][::-1]
    assert not _call(d, uns.ravel(), ptr, n)                   # unsorted row
    slf = ind.copy(); slf[7, 0] = 7; slf[7].sort()
    assert not _call(d, slf.ravel(), ptr, n)                   # self entry
    oor = ind.copy(); oor[9, 2] = n
    assert not _call(d, oor.ravel(), ptr, n)                   # column outside [0, n)


def test_workspace_from_graph_runs_as_from_host_P():
    X, G, P, _ = problem(5000, seed=8, dim=20)
    be = _be()
    Ph = be.joint_P(G.tocsr(), 30.0)
    n = Ph.shape[0]
    Y0 = O.init_embedding(n, 2, 9)
    a = Engine(Ph, Y0, n_iter=60)
    a.run_all()
    Ya, kla = a.embedding(), a.kl()
    a.close()
    Gp = be.prepare_knn_graph(G.tocsr())
    p = a.params
    p.n_iter = 60
    Yc = np.ascontiguousarray(Y0)
    from tsne_h2pack._backend import DTYPE
    p.init_method, p.init_Y = 1, Yc.ctypes.data_as(ctypes.POINTER(DTYPE))
    d, i, pt = be._graph_arrays(Gp)
    ws = be._lib.tsne_init_with_knn_distances(None, n, 0, 2, ctypes.byref(p),
                                              d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              i.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                              pt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(Gp.nnz))
    assert ws
    assert be._lib.tsne_run(ws) == 0
    Yb = np.zeros((2, n))
    be._lib.tsne_get_embedding(ws, Yb)
    klb = float(be._lib.compute_kl_divergence(ws))
    be._lib.tsne_destroy(ws)
    assert rel(Yb, Ya) < 1e-6
    assert abs(klb - kla) <= 1e-6 * abs(kla)
