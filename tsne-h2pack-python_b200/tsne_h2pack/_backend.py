"""ctypes binding of the engine's C ABI (include/tsne_h2pack.h).

Interface-compatible with the reference's loader (tsne_h2pack/_backend.py of the reference
project): the same constants, ctypes structures (TSNEParams is the 160-byte tsne_params_t),
TSNEBackend methods and CSR converters. The shared library is looked up where the reference
looks (tsne_h2pack/_lib/, then build/lib/); there is no fallback: a missing library or a
missing CUDA device raises RuntimeError.
"""
import ctypes
import os
import platform
import sys
import time
from pathlib import Path
from typing import Optional, Tuple

import numpy as np

IS_LINUX = platform.system() == "Linux"
IS_MACOS = platform.system() == "Darwin"
IS_WINDOWS = platform.system() == "Windows"

DTYPE = ctypes.c_double
NP_DTYPE = np.float64


class TSNEParams(ctypes.Structure):
    """tsne_params_t (include/tsne_h2pack.h), 160 bytes; explicit padding fields keep the
    offsets of the C layout (reference _backend.py:51-96)."""
    _fields_ = [
        ("n_iter", ctypes.c_int),                 # 0
        ("_pad1", ctypes.c_int),                  # 4
        ("perplexity", DTYPE),                    # 8
        ("learning_rate", DTYPE),                 # 16
        ("momentum", DTYPE),                      # 24
        ("initial_momentum", DTYPE),              # 32
        ("momentum_switch_iter", ctypes.c_int),   # 40
        ("_pad2", ctypes.c_int),                  # 44
        ("early_exag", DTYPE),                    # 48
        ("early_exag_iter", ctypes.c_int),        # 56
        ("use_vptree", ctypes.c_int),             # 60
        ("h2_tol", DTYPE),                        # 64
        ("h2_rebuild_freq", ctypes.c_int),        # 72
        ("h2pack_print_level", ctypes.c_int),     # 76
        ("init_method", ctypes.c_int),            # 80
        ("random_seed", ctypes.c_int),            # 84
        ("verbose", ctypes.c_int),                # 88
        ("print_freq", ctypes.c_int),             # 92
        ("enable_early_stopping", ctypes.c_int),  # 96
        ("_pad4", ctypes.c_int),                  # 100
        ("convergence_tol", DTYPE),               # 104
        ("convergence_patience", ctypes.c_int),   # 112
        ("min_iter", ctypes.c_int),               # 116
        ("sklearn_compatible", ctypes.c_int),     # 120
        ("enable_profiling", ctypes.c_int),       # 124
        ("profiling_output_file", ctypes.c_char_p),  # 128
        ("num_threads", ctypes.c_int),            # 136
        ("h2_leaf_size", ctypes.c_int),           # 140
        ("h2_rebuild_freq_early", ctypes.c_int),  # 144
        ("_pad5", ctypes.c_int),                  # 148
        ("init_Y", ctypes.POINTER(DTYPE)),        # 152 -> 160
    ]


def _optional_ndpointer(**kwargs):
    """An ndpointer argument type that also accepts None (NULL)."""
    base = np.ctypeslib.ndpointer(**kwargs)

    def from_param(cls, obj):
        return None if obj is None else base.from_param(obj)

    return type(base.__name__, (base,), {"from_param": classmethod(from_param)})


class SparseMatrix(ctypes.Structure):
    """sparse_matrix_t: CSR with int32 indices and float64 values."""
    _fields_ = [
        ("n_rows", ctypes.c_int),
        ("n_cols", ctypes.c_int),
        ("nnz", ctypes.c_int),
        ("row_ptr", ctypes.POINTER(ctypes.c_int)),
        ("col_idx", ctypes.POINTER(ctypes.c_int)),
        ("values", ctypes.POINTER(DTYPE)),
    ]


class TSNEWorkspace(ctypes.Structure):
    """Opaque workspace (only pointers to it cross the boundary)."""


def library_candidates():
    here = Path(__file__).resolve().parent
    tag = f"cpython-{sys.version_info.major}{sys.version_info.minor}-{platform.machine()}-linux-gnu"
    return [
        here / "_lib" / f"libtsne_h2pack.{tag}.so",
        here / "_lib" / "libtsne_h2pack.so",
        here.parent / "build" / "lib" / "libtsne_h2pack.so",
    ]


class TSNEBackend:
    """Loads the native engine and marshals arrays across the C ABI."""

    def __init__(self):
        if IS_WINDOWS:
            raise RuntimeError("Windows is not supported; use Linux (or WSL2) with a CUDA device.")
        self._lib = self._load_native_library()
        self._backend_type = "native"

    def _load_native_library(self):
        lib_path = next((c for c in library_candidates() if c.exists()), None)
        if lib_path is None:
            raise RuntimeError(
                "Native library not found (tsne_h2pack/_lib/libtsne_h2pack.so). Build it with "
                "`python tsne-h2pack-python_b200/build.py`.")
        try:
            lib = ctypes.CDLL(str(lib_path))
        except OSError as e:
            raise RuntimeError(f"Failed to load native library from {lib_path}: {e}")
        self._configure_ctypes_signatures(lib)
        self.library_path = lib_path
        return lib

    @staticmethod
    def _configure_ctypes_signatures(lib):
        """Argument and return types of every entry point the Python side calls
        (reference _backend.py:345-448), plus the engine's inspection calls."""
        ws_p = ctypes.POINTER(TSNEWorkspace)
        f64 = np.ctypeslib.ndpointer(dtype=NP_DTYPE, flags="C_CONTIGUOUS")
        lib.tsne_create_default_params.argtypes = []
        lib.tsne_create_default_params.restype = TSNEParams
        lib.tsne_init.argtypes = [f64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TSNEParams)]
        lib.tsne_init.restype = ws_p
        lib.tsne_init_with_P.argtypes = [
            _optional_ndpointer(dtype=NP_DTYPE, flags="C_CONTIGUOUS", ndim=2), ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.POINTER(TSNEParams), ctypes.POINTER(SparseMatrix)]
        lib.tsne_init_with_P.restype = ws_p
        lib.tsne_run.argtypes = [ws_p]
        lib.tsne_run.restype = ctypes.c_int
        lib.tsne_get_embedding.argtypes = [ws_p, f64]
        lib.tsne_get_embedding.restype = None
        lib.tsne_destroy.argtypes = [ws_p]
        lib.tsne_destroy.restype = None
        lib.tsne_fit_transform.argtypes = [f64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(TSNEParams), f64]
        lib.tsne_fit_transform.restype = ctypes.c_int
        lib.tsne_fit_transform_with_P.argtypes = [
            _optional_ndpointer(dtype=NP_DTYPE, flags="C_CONTIGUOUS", ndim=2), ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.POINTER(TSNEParams), ctypes.POINTER(SparseMatrix), f64]
        lib.tsne_fit_transform_with_P.restype = ctypes.c_int
        lib.compute_P_from_knn_distances.argtypes = [
            ctypes.POINTER(DTYPE), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_double, ctypes.c_int]
        lib.compute_P_from_knn_distances.restype = ctypes.POINTER(SparseMatrix)
        lib.sparse_matrix_destroy.argtypes = [ctypes.POINTER(SparseMatrix)]
        lib.sparse_matrix_destroy.restype = None
        lib.sparse_matrix_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.sparse_matrix_create.restype = ctypes.POINTER(SparseMatrix)
        lib.tsne_set_init_profiling_times.argtypes = [ws_p, ctypes.c_double, ctypes.c_double]
        lib.tsne_set_init_profiling_times.restype = None
        lib.compute_kl_divergence.argtypes = [ws_p]
        lib.compute_kl_divergence.restype = DTYPE
        # engine-only calls (inspection and partial runs)
        lib.tsne_run_range.argtypes = [ws_p, ctypes.c_int, ctypes.c_int]
        lib.tsne_run_range.restype = ctypes.c_int
        lib.tsne_get_state.argtypes = [ws_p, _optional_ndpointer(dtype=NP_DTYPE, flags="C_CONTIGUOUS"),
                                       _optional_ndpointer(dtype=NP_DTYPE, flags="C_CONTIGUOUS"),
                                       ctypes.POINTER(ctypes.c_double)]
        lib.tsne_get_state.restype = ctypes.c_int
        lib.tsne_set_embedding.argtypes = [ws_p, f64]
        lib.tsne_set_embedding.restype = ctypes.c_int
        lib.tsne_get_run_stats.argtypes = [ws_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]
        lib.tsne_get_run_stats.restype = ctypes.c_int
        # P built on the device
        lib.tsne_joint_P_from_knn_distances.argtypes = [
            ctypes.POINTER(DTYPE), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
            ctypes.c_int, ctypes.c_double]
        lib.tsne_joint_P_from_knn_distances.restype = ctypes.POINTER(SparseMatrix)
        lib.tsne_init_with_knn_distances.argtypes = [
            _optional_ndpointer(dtype=NP_DTYPE, flags="C_CONTIGUOUS", ndim=2), ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.POINTER(TSNEParams), ctypes.POINTER(DTYPE), ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        lib.tsne_init_with_knn_distances.restype = ws_p

    def create_default_params(self) -> TSNEParams:
        """Defaults of tsne_create_default_params, filled on the Python side (the reference
        avoids returning the struct by value on ARM64, _backend.py:450-502)."""
        p = TSNEParams()
        p.n_iter = 1000
        p.perplexity = 30.0
        p.learning_rate = -1.0
        p.momentum = 0.8
        p.initial_momentum = 0.5
        p.momentum_switch_iter = 250
        p.early_exag = 12.0
        p.early_exag_iter = 250
        p.use_vptree = 2
        p.h2_tol = 1e-3
        p.h2_rebuild_freq = 10
        p.h2pack_print_level = 0
        p.init_method = 0
        p.random_seed = -1
        p.verbose = 1
        p.print_freq = 50
        p.enable_early_stopping = 0
        p.convergence_tol = 1e-5
        p.convergence_patience = 10
        p.min_iter = 250
        p.sklearn_compatible = 1
        p.enable_profiling = 0
        p.profiling_output_file = None
        p.num_threads = 1
        p.h2_leaf_size = 100
        p.h2_rebuild_freq_early = 10
        p.init_Y = None
        return p

    def fit_transform(self, X: np.ndarray, n_components: int, params: TSNEParams) -> Tuple[np.ndarray, dict]:
        """Embed X (n_samples, n_features) through tsne_fit_transform (k-NN and P built by the
        engine). The KL divergence is not available on this path (reported as 0.0)."""
        X = np.ascontiguousarray(X, dtype=NP_DTYPE)
        n, f = X.shape
        Xc = np.ascontiguousarray(X.T)
        Yc = np.zeros((n_components, n), dtype=NP_DTYPE)
        rc = self._lib.tsne_fit_transform(Xc, n, f, n_components, params, Yc)
        if rc != 0:
            raise RuntimeError(f"tsne_fit_transform failed with code {rc}")
        return np.ascontiguousarray(Yc.T), {"kl_divergence": 0.0, "n_iter": params.n_iter}

    def fit_transform_with_P(self, X: Optional[np.ndarray], P_scipy, n_components: int,
                             params: TSNEParams) -> Tuple[np.ndarray, dict]:
        """Embed with a precomputed joint P (scipy CSR); the features are not passed down."""
        from scipy.sparse import csr_matrix
        if not isinstance(P_scipy, csr_matrix):
            raise TypeError(f"P must be scipy CSR matrix, got {type(P_scipy)}")
        n = P_scipy.shape[0]
        n_features = X.shape[1] if X is not None else 0
        P_c = scipy_csr_to_c_sparse_matrix(P_scipy, self._lib)
        Yc = np.zeros((n_components, n), dtype=NP_DTYPE)
        rc = self._lib.tsne_fit_transform_with_P(None, n, n_features, n_components, ctypes.byref(params), P_c, Yc)
        if rc != 0:
            raise RuntimeError(f"tsne_fit_transform_with_P failed with code {rc}")
        return np.ascontiguousarray(Yc.T), {"kl_divergence": 0.0, "n_iter": params.n_iter}

    def pca_init(self, X: np.ndarray, n_components: int) -> np.ndarray:
        """init='pca' on the device (tsne_pca_init): the exact PCA projection of X, scaled to a
        first-coordinate standard deviation of 1e-4 (reference manifold.py:399-416, which uses
        scikit-learn's randomized approximation of the same projection)."""
        X = np.ascontiguousarray(X, dtype=NP_DTYPE)
        n, f = X.shape
        Y = np.zeros((n, n_components), dtype=NP_DTYPE)
        self._lib.tsne_pca_init.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p]
        self._lib.tsne_pca_init.restype = ctypes.c_int
        rc = self._lib.tsne_pca_init(X.ctypes.data, n, f, int(n_components), Y.ctypes.data)
        if rc == -3:
            raise ValueError("init='pca' failed: X holds inf/NaN or has no variance along its first principal "
                             "component; pass init='random'")
        if rc != 0:
            raise RuntimeError(f"tsne_pca_init failed ({rc})")
        return Y

    def score_embedding(self, Y: np.ndarray, P, knn_graph, k: int = 10, n_eval: int = 5000, seed: int = 0) -> dict:
        """The reference's quality scores (benchmarks/quality.py:56-90) on the device
        (tsne_score_embedding): k-NN preservation of n_eval seeded queries (input-space
        neighbours: the k nearest of each row of knn_graph) and the KL divergence under P with
        the exact Z. Y: (n_samples, n_components)."""
        n, d = Y.shape
        Yc = np.ascontiguousarray(np.asarray(Y, dtype=NP_DTYPE).T)
        rng = np.random.default_rng(seed)
        q = np.ascontiguousarray(rng.choice(n, size=min(n_eval, n), replace=False), dtype=np.int32)
        G = knn_graph.tocsr()
        hd = np.empty((len(q), k), dtype=np.int32)
        for r, i in enumerate(q):
            a, b = G.indptr[i], G.indptr[i + 1]
            if b - a < k:
                raise ValueError(f"row {i} of the k-NN graph has fewer than k = {k} neighbours")
            hd[r] = G.indices[a:b][np.argsort(G.data[a:b], kind="stable")[:k]]
        Pc = scipy_csr_to_c_sparse_matrix(P.tocsr(), self._lib)
        kp, kl = ctypes.c_double(), ctypes.c_double()
        self._lib.tsne_score_embedding.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.POINTER(SparseMatrix), ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                   ctypes.POINTER(ctypes.c_double)]
        self._lib.tsne_score_embedding.restype = ctypes.c_int
        try:
            rc = self._lib.tsne_score_embedding(Yc.ctypes.data, n, d, Pc, q.ctypes.data, len(q), hd.ctypes.data, k,
                                                ctypes.byref(kp), ctypes.byref(kl))
        finally:
            self._lib.sparse_matrix_destroy(Pc)
        if rc != 0:
            raise RuntimeError(f"tsne_score_embedding failed ({rc})")
        return {"kl": kl.value, "knn_preservation": kp.value}

    def conditional_P(self, knn_distances_csr, perplexity: float, num_threads: int = 1):
        """P_j|i of a k-NN distance graph (CSR, L2 distances, rows sorted, no self entries)."""
        from scipy.sparse import csr_matrix
        n = knn_distances_csr.shape[0]
        data = np.ascontiguousarray(knn_distances_csr.data, dtype=np.float64)
        ind = np.ascontiguousarray(knn_distances_csr.indices, dtype=np.int32)
        ptr = np.ascontiguousarray(knn_distances_csr.indptr, dtype=np.int32)
        m = self._lib.compute_P_from_knn_distances(
            data.ctypes.data_as(ctypes.POINTER(DTYPE)), ind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, int(knn_distances_csr.nnz),
            ctypes.c_double(perplexity), int(num_threads))
        if not m:
            raise RuntimeError("compute_P_from_knn_distances returned NULL")
        mc = m.contents
        P = csr_matrix((np.ctypeslib.as_array(mc.values, shape=(mc.nnz,)).copy(),
                        np.ctypeslib.as_array(mc.col_idx, shape=(mc.nnz,)).copy(),
                        np.ctypeslib.as_array(mc.row_ptr, shape=(mc.n_rows + 1,)).copy()), shape=(n, n))
        self._lib.sparse_matrix_destroy(m)
        return P

    @staticmethod
    def prepare_knn_graph(knn_distances_csr):
        """Rows sorted by column and self entries dropped: the calibration sums each row in
        storage order, so every path must hand it the same order (reference
        _backend.py:651-663)."""
        from scipy.sparse import csr_matrix
        n = knn_distances_csr.shape[0]
        if not knn_distances_csr.has_sorted_indices:
            knn_distances_csr = knn_distances_csr.copy()
            knn_distances_csr.sort_indices()
        lens = np.diff(knn_distances_csr.indptr)
        if n > 0 and knn_distances_csr.nnz == n * int(lens[0]) and np.all(lens == lens[0]):
            # k entries in every row (a k-NN graph): compare in place, rows as a broadcast column
            k = int(lens[0])
            if k == 0 or not np.any(knn_distances_csr.indices.reshape(n, k) ==
                                    np.arange(n, dtype=knn_distances_csr.indices.dtype)[:, None]):
                return knn_distances_csr
        rows = np.repeat(np.arange(n, dtype=np.int32), lens)
        if np.any(knn_distances_csr.indices == rows):
            keep = knn_distances_csr.indices != rows
            knn_distances_csr = csr_matrix(
                (knn_distances_csr.data[keep], knn_distances_csr.indices[keep],
                 np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))])),
                shape=knn_distances_csr.shape)
        return knn_distances_csr

    @staticmethod
    def _graph_arrays(G):
        data = np.ascontiguousarray(G.data, dtype=NP_DTYPE)
        ind = np.ascontiguousarray(G.indices, dtype=np.int32)
        ptr = np.ascontiguousarray(G.indptr, dtype=np.int32)
        return data, ind, ptr

    def joint_P_device(self, knn_distances_csr, perplexity: float):
        """The same P as joint_P with every step on the device (tsne_joint_P_from_knn_distances):
        entries equal joint_P's bit for bit except for the normalising total's rounding."""
        from scipy.sparse import csr_matrix
        G = self.prepare_knn_graph(knn_distances_csr)
        n = G.shape[0]
        data, ind, ptr = self._graph_arrays(G)
        m = self._lib.tsne_joint_P_from_knn_distances(
            data.ctypes.data_as(ctypes.POINTER(DTYPE)), ind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, int(G.nnz), ctypes.c_double(perplexity))
        if not m:
            raise RuntimeError("tsne_joint_P_from_knn_distances returned NULL")
        mc = m.contents
        P = csr_matrix((np.ctypeslib.as_array(mc.values, shape=(mc.nnz,)).copy() if mc.nnz else np.zeros(0),
                        np.ctypeslib.as_array(mc.col_idx, shape=(mc.nnz,)).copy() if mc.nnz else
                        np.zeros(0, np.int32),
                        np.ctypeslib.as_array(mc.row_ptr, shape=(mc.n_rows + 1,)).copy()), shape=(n, n))
        self._lib.sparse_matrix_destroy(m)
        return P

    def joint_P(self, knn_distances_csr, perplexity: float, num_threads: int = 1):
        """Symmetric normalised P = (P_c + P_c^T) / sum from a k-NN distance graph (calibration
        on the device, symmetrisation on the host, as the reference's _backend.py:672-718)."""
        G = self.prepare_knn_graph(knn_distances_csr)
        Pc = self.conditional_P(G, perplexity, num_threads)
        Ps = Pc + Pc.T
        total = Ps.sum()
        if total > 0:
            Ps.data /= total
        return Ps.tocsr()

    def fit_transform_with_knn_distances(self, X: Optional[np.ndarray], knn_distances_csr, n_components: int,
                                         params: TSNEParams, init_Y: Optional[np.ndarray] = None
                                         ) -> Tuple[np.ndarray, dict]:
        """Embed from a k-NN distance graph of any source (reference _backend.py:611-781):
        P calibrated, symmetrised and normalised on the device (tsne_init_with_knn_distances:
        P never visits the host), then run -> embedding -> KL -> destroy. With the environment
        switch TSNE_HOST_P=1, P is symmetrised on the host as the reference does
        (tsne_init_with_P), which reproduces the reference package's results bit for bit."""
        from scipy.sparse import csr_matrix
        if not isinstance(knn_distances_csr, csr_matrix):
            raise TypeError(f"knn_distances must be scipy CSR matrix, got {type(knn_distances_csr)}")
        n = knn_distances_csr.shape[0]
        n_features = X.shape[1] if X is not None else 0
        t0 = time.time()
        host_P = os.environ.get("TSNE_HOST_P", "0") not in ("", "0")
        if host_P:
            P = self.joint_P(knn_distances_csr, params.perplexity, params.num_threads)
            P_c = scipy_csr_to_c_sparse_matrix(P, self._lib)
        else:
            G = self.prepare_knn_graph(knn_distances_csr)
            gdata, gind, gptr = self._graph_arrays(G)
        p_time = time.time() - t0
        knn_time = getattr(knn_distances_csr, "knn_time", 0.0)
        Yc = np.zeros((n_components, n), dtype=NP_DTYPE)
        init_c = None
        if init_Y is not None:
            init_Y = np.asarray(init_Y)
            if init_Y.shape != (n, n_components):
                raise ValueError(f"init_Y must have shape {(n, n_components)}, got {init_Y.shape}")
            init_c = np.ascontiguousarray(init_Y.T, dtype=NP_DTYPE)
            params.init_method = 1
            params.init_Y = init_c.ctypes.data_as(ctypes.POINTER(DTYPE))
        else:
            params.init_method = 0
            params.init_Y = None
        if host_P:
            ws = self._lib.tsne_init_with_P(None, n, n_features, n_components, ctypes.byref(params), P_c)
        else:
            ws = self._lib.tsne_init_with_knn_distances(
                None, n, n_features, n_components, ctypes.byref(params),
                gdata.ctypes.data_as(ctypes.POINTER(DTYPE)), gind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                gptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(G.nnz))
            p_time = time.time() - t0
        params.init_Y = None
        del init_c
        if not ws:
            raise RuntimeError("tsne_init_with_P returned NULL")
        if params.enable_profiling:
            self._lib.tsne_set_init_profiling_times(ws, ctypes.c_double(knn_time), ctypes.c_double(p_time))
        try:
            rc = self._lib.tsne_run(ws)
            if rc != 0:
                raise RuntimeError(f"tsne_run failed with code {rc}")
            self._lib.tsne_get_embedding(ws, Yc)
            kl = float(self._lib.compute_kl_divergence(ws))
        finally:
            self._lib.tsne_destroy(ws)
        return np.ascontiguousarray(Yc.T), {"kl_divergence": kl, "n_iter": params.n_iter}

    @property
    def backend_type(self) -> str:
        return self._backend_type

    def is_available(self) -> bool:
        return True


def scipy_csr_to_sparse_matrix(P_scipy) -> Tuple[SparseMatrix, dict]:
    """A SparseMatrix that borrows the arrays of a scipy CSR matrix; keep the returned dict
    alive while the struct is in use."""
    from scipy.sparse import csr_matrix
    if not isinstance(P_scipy, csr_matrix):
        raise TypeError(f"Expected scipy CSR matrix, got {type(P_scipy)}")
    arrays = {
        "row_ptr": np.ascontiguousarray(P_scipy.indptr, dtype=np.int32),
        "col_idx": np.ascontiguousarray(P_scipy.indices, dtype=np.int32),
        "values": np.ascontiguousarray(P_scipy.data, dtype=np.float64),
    }
    m = SparseMatrix()
    m.n_rows, m.n_cols = P_scipy.shape
    m.nnz = P_scipy.nnz
    m.row_ptr = arrays["row_ptr"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    m.col_idx = arrays["col_idx"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    m.values = arrays["values"].ctypes.data_as(ctypes.POINTER(DTYPE))
    return m, arrays


_copy_pool = None


def _copy(dst, src, nbytes, chunk=64 << 20):
    """memmove of a large host array in chunks on a few threads (ctypes releases the GIL during
    the copy), so that filling a C matrix of 10^8 entries is not bound by one core."""
    global _copy_pool
    if nbytes < 4 * chunk:
        ctypes.memmove(dst, src, nbytes)
        return
    if _copy_pool is None:
        from concurrent.futures import ThreadPoolExecutor
        _copy_pool = ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1))
    dst, src = ctypes.cast(dst, ctypes.c_void_p).value, ctypes.cast(src, ctypes.c_void_p).value
    jobs = [_copy_pool.submit(ctypes.memmove, dst + o, src + o, min(chunk, nbytes - o))
            for o in range(0, nbytes, chunk)]
    for j in jobs:
        j.result()


def scipy_csr_to_c_sparse_matrix(P_scipy, lib) -> "ctypes.POINTER(SparseMatrix)":
    """A C-allocated copy (sparse_matrix_create) that tsne_init_with_P may take over."""
    from scipy.sparse import csr_matrix
    if not isinstance(P_scipy, csr_matrix):
        raise TypeError(f"Expected scipy CSR matrix, got {type(P_scipy)}")
    n_rows, n_cols = P_scipy.shape
    ptr = lib.sparse_matrix_create(n_rows, n_cols, P_scipy.nnz)
    if not ptr:
        raise MemoryError("Failed to allocate sparse matrix in C")
    m = ptr.contents
    rp = np.ascontiguousarray(P_scipy.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(P_scipy.indices, dtype=np.int32)
    pv = np.ascontiguousarray(P_scipy.data, dtype=np.float64)
    _copy(m.row_ptr, rp.ctypes.data, rp.nbytes)
    if P_scipy.nnz:
        _copy(m.col_idx, ci.ctypes.data, ci.nbytes)
        _copy(m.values, pv.ctypes.data, pv.nbytes)
    return ptr


_backend: Optional[TSNEBackend] = None


def get_backend() -> TSNEBackend:
    """The process-wide backend (loaded on first use)."""
    global _backend
    if _backend is None:
        _backend = TSNEBackend()
    return _backend
