"""The 3D bases (recomputed-row interpolative decompositions) across their CTA size classes.

The 3D basis kernel takes a node's candidate rows in one of three CTA sizes: leaves of at most
32 points, leaves of 33-128 points, and internal nodes with leaves above 128 points; leaves
above 512 points (only at the key depth) take the stored-matrix kernel. On clustered 3D
embeddings (Zipf-sized Gaussian blobs, 20,000 points) with leaf sizes 40 and 300 and a block
of 600 coincident points (whose leaf sends every leaf to the stored-matrix kernel), the device tree, node table and lists equal the oracle's bit for bit,
and the H2 force and Z are within h2_tol (1e-2) of the FP64 exact sums, as in
test_gpu_engine.py. The stored-matrix kernel (TSNE_ID3=0) on the same embedding gives a force
within h2_tol as well, and the two differ by less than h2_tol.
"""
import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, rel2

pytestmark = pytest.mark.gpu

N = 20_000
TOL = 1e-2


def _blobs(n, seed):
    """(3, n) Zipf-sized Gaussian blobs, stored at float precision."""
    rng = np.random.default_rng(seed)
    k = 24
    w = np.arange(1, k + 1, dtype=np.float64) ** -1.1
    counts = rng.multinomial(n, w / w.sum())
    centres = rng.uniform(-40.0, 40.0, size=(k, 3))
    lab = np.repeat(np.arange(k), counts)
    Y = centres[lab] + rng.normal(scale=1.5, size=(n, 3))
    return np.ascontiguousarray(Y.T).astype(np.float32).astype(np.float64)


def _ring(n):
    i = np.arange(n)
    P = csr_matrix((np.full(2 * n, 0.5 / n), (np.concatenate([i, (i + 1) % n]), np.concatenate([(i + 1) % n, i]))),
                   shape=(n, n))
    P.sort_indices()
    return P


def _check(Y, leaf):
    """Tree and lists against the oracle, force and Z against the FP64 exact sums; returns the
    leaf sizes and the device force."""
    P = _ring(Y.shape[1])
    eng = Engine(P, Y, n_iter=1, h2_leaf_size=leaf, h2_tol=TOL)
    assert eng.rebuild() == 0
    dev = eng.h2()
    assert dev is not None, "the tree is too shallow for an H2 matrix"
    h = O.H2(Y, leaf_size=leaf, tol=TOL)
    np.testing.assert_array_equal(h.perm(), dev["perm"])
    on = h.nodes()
    for k in on:
        np.testing.assert_array_equal(on[k], dev["nodes"][k], err_msg=k)
    fp, fi, np_, ni = h.lists()
    np.testing.assert_array_equal(fi, dev["far_idx"])
    np.testing.assert_array_equal(ni, dev["near_idx"])
    sizes = (on["end"] - on["start"])[(on["is_leaf"] == 1) & (on["level"] >= 2)]
    F, Z = eng.repulsive(Y)
    eng.close()
    s, v = O.exact_sv(Y)
    Ze, Fe = O.z_force(Y, s, v)
    ferr, zerr = rel2(F, Fe), abs(Z - Ze) / Ze
    print(f"3D leaf {leaf}: leaves {len(sizes)}, largest {sizes.max()}, force rel {ferr:.3e}, Z rel {zerr:.3e}")
    assert ferr <= TOL
    assert zerr <= TOL
    return sizes, F


def test_small_leaves():
    """leaf_size 40: leaves of the 128-thread (at most 32 points) and 256-thread CTAs."""
    sizes, _ = _check(_blobs(N, 1), 40)
    assert sizes.max() <= 40 and (sizes <= 32).any() and (sizes > 32).any()


def test_large_leaves():
    """leaf_size 300: all three CTA sizes (leaves above 128 points take the 512-thread one)."""
    sizes, _ = _check(_blobs(N, 2), 300)
    assert (sizes <= 32).any() and ((sizes > 32) & (sizes <= 128)).any() and (sizes > 128).any()


def test_coincident_points_above_512():
    """600 points at one position: a leaf at the key depth above 512 points. The leaves' bases
    then come from the stored-matrix kernel; the internal nodes keep the recomputed rows."""
    Y = _blobs(N, 3)
    idx = np.random.default_rng(7).choice(N, 600, replace=False)
    Y[:, idx] = Y[:, idx[:1]]
    sizes, _ = _check(Y, 100)
    assert sizes.max() >= 600


def test_recomputed_rows_match_stored_matrix(monkeypatch):
    """The stored-matrix kernel (TSNE_ID3=0) on the same embedding: both forces within h2_tol of
    the exact sums and of each other."""
    Y = _blobs(N, 4)
    _, F_new = _check(Y, 100)
    monkeypatch.setenv("TSNE_ID3", "0")
    _, F_old = _check(Y, 100)
    diff = rel2(F_new, F_old)
    print(f"recomputed rows vs stored matrix: force rel {diff:.3e}")
    assert diff <= TOL
