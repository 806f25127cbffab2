"""Leaf-size autotuner of the H2 matrix per size bucket (no counterpart in the reference, whose
`h2_leaf_size` is the user's parameter, default 100).

The leaf size trades the near field (leaf x leaf blocks, FP32 pair kernels) against the tree,
the lists and the bases (more, smaller nodes); where the balance lies depends on N and on the
GPU. For a bucket of sizes (powers of two) the tuner builds a workspace on a synthetic
embedding shaped like a late t-SNE state (Zipf-sized Gaussian blobs spread over a square whose
side grows as sqrt(N)), runs rebuild iterations of the engine for each candidate leaf size and
keeps the one with the smallest device time per iteration (the engine's CUDA-event timer).
Every candidate keeps the repulsive force within h2_tol (the interpolative decompositions stop
at the same relative tolerance whatever the leaf size), so the choice trades time only; the
result differs from the default leaf size's by rounding-level changes of the H2 matrix, within
h2_tol.

    >>> from tsne_h2pack.autotune import LeafTuner
    >>> tuner = LeafTuner()
    >>> tuner.leaf_for(20000, 2)          # measured once per (dimension, bucket), then cached
"""
import ctypes
import math

import numpy as np
from scipy.sparse import csr_matrix

from ._backend import DTYPE, TSNEWorkspace, get_backend, scipy_csr_to_c_sparse_matrix

CANDIDATES = (48, 64, 100, 128, 160)


def bucket_of(n):
    """The size bucket of n: floor(log2 n)."""
    return int(math.floor(math.log2(max(2, n))))


def synthetic_embedding(n, d, seed=0):
    """(d, n) Zipf-sized Gaussian blobs over a square of side 0.4 sqrt(n), blob spread 2% of it
    (the shape of a converged t-SNE embedding at this N)."""
    rng = np.random.default_rng(seed)
    k = int(min(100, max(5, n // 2000)))
    w = np.arange(1, k + 1, dtype=np.float64) ** -1.1
    counts = rng.multinomial(n, w / w.sum())
    side = 0.4 * math.sqrt(n)
    centres = rng.uniform(-side / 2, side / 2, size=(k, d))
    lab = np.repeat(np.arange(k), counts)
    return np.ascontiguousarray((centres[lab] + rng.normal(scale=0.02 * side, size=(n, d))).T)


def _ring_P(n):
    i = np.arange(n)
    rows = np.concatenate([i, (i + 1) % n])
    cols = np.concatenate([(i + 1) % n, i])
    P = csr_matrix((np.full(2 * n, 0.5 / n), (rows, cols)), shape=(n, n))
    P.sort_indices()
    return P


def time_leaf(n, d, leaf, h2_tol, iters=3, seed=0):
    """Device ms per rebuild iteration (H2 rebuild + product + attractive pass of a ring P) at
    this leaf size, on the synthetic embedding."""
    be = get_backend()
    lib = be._lib
    lib.tsne_get_timing.argtypes = [ctypes.POINTER(TSNEWorkspace), ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    Y0 = synthetic_embedding(n, d, seed)
    p = be.create_default_params()
    p.n_iter, p.verbose = 20, 0
    p.h2_tol, p.h2_leaf_size = h2_tol, int(leaf)
    p.h2_rebuild_freq, p.h2_rebuild_freq_early = 3, 10
    p.learning_rate = 1e-9                      # the embedding stays put while the rebuilds are timed
    p.init_method, p.init_Y = 1, Y0.ctypes.data_as(ctypes.POINTER(DTYPE))
    ws = lib.tsne_init_with_P(None, n, 0, d, ctypes.byref(p), scipy_csr_to_c_sparse_matrix(_ring_P(n), lib))
    p.init_Y = None
    if not ws:
        raise RuntimeError("autotune: tsne_init_with_P failed")
    try:
        if lib.tsne_run_range(ws, 1, 2) != 0:       # warm-up (iterations below 20 rebuild every time)
            raise RuntimeError("autotune: run failed")
        if lib.tsne_run_range(ws, 2, 2 + iters) != 0:
            raise RuntimeError("autotune: run failed")
        run_ms, a_ms, a_n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        lib.tsne_get_timing(ws, ctypes.byref(run_ms), ctypes.byref(a_ms), ctypes.byref(a_n))
        return run_ms.value / iters
    finally:
        lib.tsne_destroy(ws)


class LeafTuner:
    """Per (dimension, size bucket) leaf size, measured on first use and cached."""

    def __init__(self, candidates=CANDIDATES, h2_tol=None):
        self.candidates = tuple(int(c) for c in candidates)
        self.h2_tol = h2_tol
        self.table = {}
        self.timings = {}

    def leaf_for(self, n, d, h2_tol=None):
        if n < 2000:
            return 100                          # the exact path: no H2 matrix
        key = (int(d), bucket_of(n))
        if key not in self.table:
            tol = h2_tol or self.h2_tol or (1e-2 if d == 2 else 3e-2)
            nb = 1 << key[1]                    # the bucket's lower end
            times = {c: time_leaf(nb, d, c, tol) for c in self.candidates}
            self.timings[key] = times
            self.table[key] = min(times, key=times.get)
        return self.table[key]
