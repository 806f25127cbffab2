"""k-NN graph front end: `get_knn_method(name).compute(X, k, n_jobs, ...)` returns a scipy CSR
matrix of L2 distances (self excluded), the contract of the reference's _knn_methods.py.

The graph is built once per fit, outside the optimisation phase this package accelerates;
'exact' and 'balltree' use scikit-learn, 'cuda' the engine's exact device scan
(tsne_knn_graph), 'pynndescent' / 'faiss' / 'annoy' use those libraries when they are
installed. Below 10K samples 'pynndescent' switches to the exact
graph, as the reference does.
"""
import time

import numpy as np


class _KNN:
    name = "base"

    def compute(self, X, k, n_jobs=1, verbose=False, **params):
        t0 = time.time()
        G = self._graph(np.asarray(X), int(k), n_jobs, verbose, **params)
        G.sort_indices()
        G.knn_time = time.time() - t0
        return G


class ExactKNN(_KNN):
    name = "exact"

    def _graph(self, X, k, n_jobs, verbose, **params):
        from sklearn.neighbors import NearestNeighbors
        nn = NearestNeighbors(n_neighbors=k, algorithm="brute", n_jobs=n_jobs, **params).fit(X)
        return nn.kneighbors_graph(mode="distance")


class CudaKNN(_KNN):
    """The exact graph on the device (tsne_knn_graph: tensor-core distance tiles, candidates
    re-ranked by exact FP32 distances; the CUDA-core scan above 64 dimensions; rows sorted by index);
    the same neighbours as 'exact' except where two distances tie to single precision."""
    name = "cuda"

    def _graph(self, X, k, n_jobs, verbose, **params):
        import ctypes
        from scipy.sparse import csr_matrix
        from ._backend import get_backend
        lib = get_backend()._lib
        Xf = np.ascontiguousarray(X, dtype=np.float32)
        n, f = Xf.shape
        idx = np.zeros((n, k), dtype=np.int32)
        dist = np.zeros((n, k), dtype=np.float32)
        lib.tsne_knn_graph.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p]
        lib.tsne_knn_graph.restype = ctypes.c_int
        rc = lib.tsne_knn_graph(Xf.ctypes.data, n, f, k, idx.ctypes.data, dist.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"tsne_knn_graph failed ({rc}): k must be in [1, min(n - 1, 256)] and a CUDA "
                               "device present")
        return csr_matrix((dist.astype(np.float64).ravel(), idx.ravel(), np.arange(0, (n + 1) * k, k)),
                          shape=(n, n))


class BallTreeKNN(_KNN):
    name = "balltree"

    def _graph(self, X, k, n_jobs, verbose, **params):
        from sklearn.neighbors import NearestNeighbors
        nn = NearestNeighbors(n_neighbors=k, algorithm="ball_tree", n_jobs=n_jobs, **params).fit(X)
        return nn.kneighbors_graph(mode="distance")


class PyNNDescentKNN(_KNN):
    name = "pynndescent"

    def _graph(self, X, k, n_jobs, verbose, **params):
        if X.shape[0] < 10000:
            return ExactKNN()._graph(X, k, n_jobs, verbose)
        try:
            from pynndescent import NNDescent
        except ImportError as e:
            raise ImportError("knn_method='pynndescent' needs the pynndescent package; pass "
                              "knn_method='exact' or install pynndescent") from e
        from scipy.sparse import csr_matrix
        index = NNDescent(X, n_neighbors=k + 1, n_jobs=n_jobs, verbose=verbose, **params)
        idx, dist = index.neighbor_graph
        n = X.shape[0]
        rows, cols, vals = [], [], []
        for i in range(n):
            keep = idx[i] != i
            sel_i, sel_d = idx[i][keep][:k], dist[i][keep][:k]
            rows.append(np.full(len(sel_i), i)); cols.append(sel_i); vals.append(sel_d)
        return csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


class FAISSKNN(_KNN):
    name = "faiss"

    def _graph(self, X, k, n_jobs, verbose, **params):
        try:
            import faiss  # noqa: F401
        except ImportError as e:
            raise ImportError("knn_method='faiss' needs the faiss package") from e
        raise NotImplementedError("knn_method='faiss' is not available in this package; use 'exact'")


class AnnoyKNN(_KNN):
    name = "annoy"

    def _graph(self, X, k, n_jobs, verbose, **params):
        try:
            import annoy  # noqa: F401
        except ImportError as e:
            raise ImportError("knn_method='annoy' needs the annoy package") from e
        raise NotImplementedError("knn_method='annoy' is not available in this package; use 'exact'")


_METHODS = {c.name: c for c in (ExactKNN, CudaKNN, BallTreeKNN, PyNNDescentKNN, FAISSKNN, AnnoyKNN)}


def list_knn_methods():
    return sorted(_METHODS)


def get_knn_method(name):
    if name not in _METHODS:
        raise ValueError(f"Unknown k-NN method '{name}'. Available: {', '.join(list_knn_methods())}")
    return _METHODS[name]()
