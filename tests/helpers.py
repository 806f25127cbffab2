"""Shared test helpers: seeded problems and a thin driver of the engine's C ABI."""
import ctypes

import numpy as np
from scipy.sparse import csr_matrix

import oracle as O
from tsne_h2pack._synthetic import knn_graph, mixture_equal, symmetric_P


def problem(n, seed=0, k=90, perplexity=30.0, dim=50, n_clusters=10):
    """Gaussian mixture -> exact k-NN graph -> joint P (oracle calibration)."""
    X, lab = mixture_equal(n, n_clusters=n_clusters, dim=dim, seed=seed)
    G = knn_graph(X, min(k, n - 1))
    G.sort_indices()
    Pc = O.conditional_P(G.data, G.indptr, perplexity, nthreads=O.nthreads_default())
    P = symmetric_P(csr_matrix((Pc, G.indices, G.indptr), shape=G.shape))
    return X, G, P, lab


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def rel2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def knn_preservation(X, Y, k=30):
    from sklearn.neighbors import NearestNeighbors
    a = NearestNeighbors(n_neighbors=k).fit(X).kneighbors(return_distance=False)
    b = NearestNeighbors(n_neighbors=k).fit(Y).kneighbors(return_distance=False)
    return float(np.mean([len(set(x) & set(y)) for x, y in zip(a, b)]) / k)


class Engine:
    """One workspace of the engine, created through tsne_init_with_P."""

    def __init__(self, P, Y0, n_iter=1000, learning_rate=None, h2_tol=1e-2, h2_rebuild_freq=3,
                 h2_rebuild_freq_early=10, h2_leaf_size=100, exact=False, **extra):
        from tsne_h2pack._backend import DTYPE, get_backend, scipy_csr_to_c_sparse_matrix
        self.be = get_backend()
        self.lib = self.be._lib
        _bind_inspection(self.lib)
        d, n = Y0.shape
        self.d, self.n = d, n
        p = self.be.create_default_params()
        p.n_iter = n_iter
        p.verbose = 0
        p.learning_rate = learning_rate or max(n / 12.0, 200.0)
        p.h2_tol = 1e-4 if exact else h2_tol
        p.h2_rebuild_freq = 999999 if exact else h2_rebuild_freq
        p.h2_rebuild_freq_early = max(h2_rebuild_freq_early, p.h2_rebuild_freq)
        p.h2_leaf_size = h2_leaf_size
        for k, v in extra.items():
            setattr(p, k, v)
        self._Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
        p.init_method = 1
        p.init_Y = self._Y0.ctypes.data_as(ctypes.POINTER(DTYPE))
        self.params = p
        Pc = scipy_csr_to_c_sparse_matrix(P.tocsr(), self.lib)
        self.ws = self.lib.tsne_init_with_P(None, n, 0, d, ctypes.byref(p), Pc)
        p.init_Y = None
        if not self.ws:
            raise RuntimeError("tsne_init_with_P returned NULL")

    def run(self, begin=0, end=None):
        end = self.params.n_iter if end is None else end
        rc = self.lib.tsne_run_range(self.ws, begin, end)
        if rc != 0:
            raise RuntimeError(f"tsne_run_range failed ({rc})")

    def run_all(self):
        rc = self.lib.tsne_run(self.ws)
        if rc != 0:
            raise RuntimeError(f"tsne_run failed ({rc})")

    def embedding(self):
        Y = np.zeros((self.d, self.n))
        self.lib.tsne_get_embedding(self.ws, Y)
        return Y

    def state(self):
        Y = np.zeros((self.d, self.n)); R = np.zeros((self.d, self.n)); z = ctypes.c_double(0)
        self.lib.tsne_get_state(self.ws, Y, R, ctypes.byref(z))
        return Y, R, z.value

    def set_embedding(self, Y):
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        assert self.lib.tsne_set_embedding(self.ws, Y) == 0

    def kl(self):
        return float(self.lib.compute_kl_divergence(self.ws))

    def rebuild(self):
        return self.lib.update_h2_matrix(self.ws, 1)

    def h2(self):
        h = self.lib.tsne_get_h2_matrix(self.ws)
        if not h:
            return None
        nn, ml, nf, nr = (ctypes.c_int() for _ in range(4))
        self.lib.tsne_h2_info(h, ctypes.byref(nn), ctypes.byref(ml), ctypes.byref(nf), ctypes.byref(nr))
        m = nn.value
        perm = np.zeros(self.n, np.int32); corner = np.zeros(3); rad = ctypes.c_double()
        self.lib.tsne_h2_get_tree(h, perm, corner, ctypes.byref(rad))
        nodes = {k: np.zeros(m, np.int32) for k in ("start", "end", "level", "parent", "first_child",
                                                    "n_child", "is_leaf")}
        self.lib.tsne_h2_get_nodes(h, *nodes.values())
        fp = np.zeros(m + 1, np.int32); fi = np.zeros(max(nf.value, 1), np.int32)
        npt = np.zeros(m + 1, np.int32); ni = np.zeros(max(nr.value, 1), np.int32)
        self.lib.tsne_h2_get_lists(h, fp, fi, npt, ni)
        rk = np.zeros(m, np.int32)
        self.lib.tsne_h2_get_ranks(h, rk)
        return dict(n_node=m, max_level=ml.value, perm=perm, corner=corner[: self.d], radius=rad.value,
                    nodes=nodes, far_ptr=fp, far_idx=fi[: nf.value], near_ptr=npt, near_idx=ni[: nr.value],
                    ranks=rk, handle=h)

    def repulsive(self, Y):
        """grad -= F for the workspace's H2 matrix (or exact sums), via the C ABI; returns (F, Z)."""
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        grad = np.zeros_like(Y)
        h = self.lib.tsne_get_h2_matrix(self.ws)
        Z = self.lib.compute_repulsive_forces_h2pack(h, Y, self.d, self.n, self.ws, grad, 0)
        return -grad, Z

    def matmul(self, cols):
        """W X of the workspace's H2 matrix for general columns (tsne_h2_matmul, diagonal
        included), original point order; cols: sequence of length-n arrays."""
        h = self.lib.tsne_get_h2_matrix(self.ws)
        X = [np.ascontiguousarray(c, dtype=np.float64) for c in cols]
        Yo = [np.zeros(self.n) for _ in X]
        xp = (ctypes.c_void_p * len(X))(*[x.ctypes.data for x in X])
        yp = (ctypes.c_void_p * len(X))(*[y.ctypes.data for y in Yo])
        assert self.lib.tsne_h2_matmul(h, len(X), xp, yp, None) == 0
        return np.array(Yo)

    def stats(self):
        nr = ctypes.c_int(); nl = ctypes.c_longlong()
        self.lib.tsne_get_run_stats(self.ws, ctypes.byref(nr), ctypes.byref(nl))
        return nr.value, nl.value

    def close(self):
        if self.ws:
            self.lib.tsne_destroy(self.ws)
            self.ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_bound = set()


def _bind_inspection(lib):
    if id(lib) in _bound:
        return
    i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    from tsne_h2pack._backend import TSNEWorkspace
    ws_p = ctypes.POINTER(TSNEWorkspace)
    lib.tsne_get_h2_matrix.argtypes = [ws_p]
    lib.tsne_get_h2_matrix.restype = ctypes.c_void_p
    lib.tsne_h2_info.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 4
    lib.tsne_h2_get_tree.argtypes = [ctypes.c_void_p, i32, f64, ctypes.POINTER(ctypes.c_double)]
    lib.tsne_h2_get_nodes.argtypes = [ctypes.c_void_p] + [i32] * 7
    lib.tsne_h2_get_lists.argtypes = [ctypes.c_void_p] + [i32] * 4
    lib.tsne_h2_get_ranks.argtypes = [ctypes.c_void_p, i32]
    lib.update_h2_matrix.argtypes = [ws_p, ctypes.c_int]
    lib.update_h2_matrix.restype = ctypes.c_int
    lib.compute_repulsive_forces_h2pack.argtypes = [ctypes.c_void_p, f64, ctypes.c_int, ctypes.c_int, ws_p, f64,
                                                    ctypes.c_int]
    lib.compute_repulsive_forces_h2pack.restype = ctypes.c_double
    lib.compute_attractive_forces.argtypes = [ctypes.c_void_p, f64, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                              f64, ctypes.c_int]
    lib.compute_attractive_forces.restype = None
    lib.tsne_h2_matmul.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                   ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]
    lib.tsne_h2_matmul.restype = ctypes.c_int
    _bound.add(id(lib))


def exact_Z_torch(Y, rows_per_block=512):
    """Z = sum_{i != j} (1 + |y_i - y_j|^2)^-1 over all pairs, in FP64 on the GPU with torch (a
    plain pairwise sum, independent of the engine; checked against the oracle's exact Z in
    the tests). Y: (d, n)."""
    import torch
    Yt = torch.tensor(np.ascontiguousarray(np.asarray(Y, dtype=np.float64).T), device="cuda")
    n = Yt.shape[0]
    sq = (Yt * Yt).sum(1)
    total = torch.zeros((), dtype=torch.float64, device="cuda")
    for s in range(0, n, rows_per_block):
        blk = Yt[s:s + rows_per_block]
        r2 = torch.addmm(sq[None, :], blk, Yt.T, beta=1.0, alpha=-2.0)
        r2 += sq[s:s + rows_per_block, None] + 1.0
        total += r2.clamp_(min=1.0).reciprocal_().sum()
        total -= blk.shape[0]          # the diagonal: r = 0 contributes 1 per row
    return float(total.item())
