"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the product never imports this module. Arrays follow the reference layout:
embeddings are (d, n) dimension-major float64, P is CSR with int32 indices.

Two native libraries back it:
  _build/liboracle.so   this project's C restatement (tsne_oracle.c)
  _ref/libtsne_ref.so   the reference's own sources compiled against ref_shim/: its exact
                        repulsion path, and its H2 product and force code run on a matrix
                        the oracle built (absent when the reference was not available at
                        build time)
"""
import ctypes
import time
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_ORA_PATH = _HERE / "_build" / "liboracle.so"
_REF_PATH = _HERE / "_ref" / "libtsne_ref.so"

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def _p(a, t):
    return a.ctypes.data_as(t)


class RunParams(ctypes.Structure):
    _fields_ = [
        ("n_iter", ctypes.c_int), ("learning_rate", ctypes.c_double),
        ("momentum", ctypes.c_double), ("initial_momentum", ctypes.c_double),
        ("momentum_switch_iter", ctypes.c_int), ("early_exag", ctypes.c_double),
        ("early_exag_iter", ctypes.c_int), ("h2_tol", ctypes.c_double),
        ("h2_rebuild_freq", ctypes.c_int), ("h2_rebuild_freq_early", ctypes.c_int),
        ("h2_leaf_size", ctypes.c_int), ("use_h2", ctypes.c_int), ("rep_reuse", ctypes.c_int),
        ("reorder", ctypes.c_int), ("nthreads", ctypes.c_int), ("iter_begin", ctypes.c_int),
        ("iter_end", ctypes.c_int),
    ]


class State(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("d", ctypes.c_int), ("rp", _i32p), ("ci", _i32p), ("pv", _f64p),
        ("Y", _f64p), ("uY", _f64p), ("gains", _f64p), ("rep", _f64p), ("rep_Z", ctypes.c_double),
        ("kl", ctypes.c_double), ("rep_valid", ctypes.c_int), ("point_order", _i32p),
        ("h2", ctypes.c_void_p), ("next_reorder", ctypes.c_int), ("n_rebuild", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _ORA_PATH.exists():
            raise RuntimeError(f"oracle library missing: {_ORA_PATH} (run `make -C oracle`)")
        L = ctypes.CDLL(str(_ORA_PATH))
        L.ora_conditional_P.argtypes = [_f64p, _i32p, ctypes.c_int, ctypes.c_double, _f64p, ctypes.c_int]
        L.ora_init_embedding.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, ctypes.c_uint]
        L.ora_exact_sv.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, _f64p, _f64p, ctypes.c_int]
        L.ora_exact_rows.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, _f64p, _f64p,
                                     ctypes.c_int]
        L.ora_z_force.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, _f64p, _f64p, _f64p]
        L.ora_z_force.restype = ctypes.c_double
        L.ora_attractive.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p,
                                     ctypes.c_double, _f64p, ctypes.c_int]
        L.ora_kl.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p,
                             ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ora_kl.restype = ctypes.c_double
        L.ora_h2_build.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, _i32p]
        L.ora_h2_build.restype = ctypes.c_void_p
        L.ora_h2_free.argtypes = [ctypes.c_void_p]
        L.ora_h2_product.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p, ctypes.c_int]
        for name in ("ora_h2_n_node", "ora_h2_max_level", "ora_h2_tree_depth", "ora_h2_n_far",
                     "ora_h2_n_near"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
            getattr(L, name).restype = ctypes.c_int
        L.ora_h2_root.argtypes = [ctypes.c_void_p, _f64p, _f64p]
        L.ora_h2_perm.argtypes = [ctypes.c_void_p]
        L.ora_h2_perm.restype = _i32p
        L.ora_h2_keys.argtypes = [ctypes.c_void_p]
        L.ora_h2_keys.restype = _u64p
        L.ora_h2_nodes.argtypes = [ctypes.c_void_p] + [_i32p] * 7
        L.ora_h2_lists.argtypes = [ctypes.c_void_p] + [_i32p] * 4
        L.ora_h2_ranks.argtypes = [ctypes.c_void_p, _i32p]
        L.ora_h2_bases.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p]
        L.ora_h2_U.argtypes = [ctypes.c_void_p]
        L.ora_h2_U.restype = _f64p
        L.ora_h2_skel.argtypes = [ctypes.c_void_p]
        L.ora_h2_skel.restype = _f64p
        L.ora_h2_n_proxy.argtypes = [ctypes.c_int]
        L.ora_h2_n_proxy.restype = ctypes.c_int
        L.ora_h2_proxies.argtypes = [ctypes.c_int, ctypes.c_double, _f64p]
        L.ora_state_create.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _f64p, _f64p]
        L.ora_state_create.restype = ctypes.POINTER(State)
        L.ora_state_free.argtypes = [ctypes.POINTER(State)]
        L.ora_run.argtypes = [ctypes.POINTER(State), ctypes.POINTER(RunParams)]
        L.ora_run.restype = ctypes.c_int
        L.ora_get_embedding.argtypes = [ctypes.POINTER(State), _f64p]
        L.ora_renumber.argtypes = [ctypes.POINTER(State), _i32p]
        _lib = L
    return _lib


def nthreads_default():
    return max(1, os.cpu_count() or 1)


# ---------------------------------------------------------------------------------------
def conditional_P(dist, indptr, perplexity, nthreads=1):
    dist = np.ascontiguousarray(dist, dtype=np.float64)
    indptr = np.ascontiguousarray(indptr, dtype=np.int32)
    out = np.zeros_like(dist)
    rc = lib().ora_conditional_P(_p(dist, _f64p), _p(indptr, _i32p), len(indptr) - 1,
                                 float(perplexity), _p(out, _f64p), int(nthreads))
    if rc != 0:
        raise ValueError("ora_conditional_P failed")
    return out


def init_embedding(n, d, seed):
    Y = np.zeros((d, n), dtype=np.float64)
    lib().ora_init_embedding(_p(Y, _f64p), n, d, ctypes.c_uint(seed & 0xFFFFFFFF))
    return Y


def exact_sv(Y, nthreads=None):
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    d, n = Y.shape
    s = np.zeros(n); v = np.zeros((d, n))
    lib().ora_exact_sv(_p(Y, _f64p), n, d, _p(s, _f64p), _p(v, _f64p), nthreads or nthreads_default())
    return s, v


def exact_rows(Y, rows, nthreads=None):
    """Exact off-diagonal sums for the points `rows` only: s (m,), v (d, m)."""
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    d, n = Y.shape
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    m = len(rows)
    s = np.zeros(m); v = np.zeros((d, m))
    lib().ora_exact_rows(_p(Y, _f64p), n, d, _p(rows, _i32p), m, _p(s, _f64p), _p(v, _f64p),
                         nthreads or nthreads_default())
    return s, v


def z_force(Y, s, v):
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    d, n = Y.shape
    s = np.ascontiguousarray(s, dtype=np.float64); v = np.ascontiguousarray(v, dtype=np.float64)
    F = np.zeros((d, n))
    Z = lib().ora_z_force(_p(Y, _f64p), n, d, _p(s, _f64p), _p(v, _f64p), _p(F, _f64p))
    return Z, F


def attractive(P, Y, exag, nthreads=None):
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    d, n = Y.shape
    rp = np.ascontiguousarray(P.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(P.indices, dtype=np.int32)
    pv = np.ascontiguousarray(P.data, dtype=np.float64)
    out = np.zeros((d, n))
    lib().ora_attractive(n, d, _p(rp, _i32p), _p(ci, _i32p), _p(pv, _f64p), _p(Y, _f64p),
                         float(exag), _p(out, _f64p), nthreads or nthreads_default())
    return out


def kl(P, Y, exag, Z, nthreads=None):
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    d, n = Y.shape
    rp = np.ascontiguousarray(P.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(P.indices, dtype=np.int32)
    pv = np.ascontiguousarray(P.data, dtype=np.float64)
    return lib().ora_kl(n, d, _p(rp, _i32p), _p(ci, _i32p), _p(pv, _f64p), _p(Y, _f64p),
                        float(exag), float(Z), nthreads or nthreads_default())


class H2:
    """Host H2 matrix of (1 + r^2)^-2 over the points Y (d, n)."""

    def __init__(self, Y, leaf_size=100, tol=1e-2, nthreads=None):
        self.Y = np.ascontiguousarray(Y, dtype=np.float64)
        self.d, self.n = self.Y.shape
        st = ctypes.c_int(0)
        self._h = lib().ora_h2_build(_p(self.Y, _f64p), self.n, self.d, int(leaf_size), float(tol),
                                     nthreads or nthreads_default(), ctypes.byref(st))
        self.status = st.value
        if not self._h:
            raise ValueError(f"ora_h2_build failed (status {self.status})")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_h2_free(self._h)
            self._h = None

    @property
    def n_node(self):
        return lib().ora_h2_n_node(self._h)

    @property
    def max_level(self):
        return lib().ora_h2_max_level(self._h)

    def root(self):
        c = np.zeros(3); r = ctypes.c_double(0)
        lib().ora_h2_root(self._h, _p(c, _f64p), ctypes.byref(r))
        return c[: self.d], r.value

    def perm(self):
        return np.ctypeslib.as_array(lib().ora_h2_perm(self._h), shape=(self.n,)).copy()

    def keys(self):
        return np.ctypeslib.as_array(lib().ora_h2_keys(self._h), shape=(self.n,)).copy()

    def nodes(self):
        m = self.n_node
        arrs = [np.zeros(m, dtype=np.int32) for _ in range(7)]
        lib().ora_h2_nodes(self._h, *[_p(a, _i32p) for a in arrs])
        keys = ("start", "end", "level", "parent", "first_child", "n_child", "is_leaf")
        return dict(zip(keys, arrs))

    def lists(self):
        m = self.n_node
        nf, nn_ = lib().ora_h2_n_far(self._h), lib().ora_h2_n_near(self._h)
        fp = np.zeros(m + 1, np.int32); fi = np.zeros(max(nf, 1), np.int32)
        np_ = np.zeros(m + 1, np.int32); ni = np.zeros(max(nn_, 1), np.int32)
        lib().ora_h2_lists(self._h, _p(fp, _i32p), _p(fi, _i32p), _p(np_, _i32p), _p(ni, _i32p))
        return fp, fi[:nf], np_, ni[:nn_]

    def ranks(self):
        r = np.zeros(self.n_node, np.int32)
        lib().ora_h2_ranks(self._h, _p(r, _i32p))
        return r

    def bases(self):
        """(ncand, skel_off, U_off, U, skel): per node the candidate rows of its U block,
        offsets of its skeleton points and of its U block (n_node + 1 entries each); U blocks
        are ncand x rank row-major, skeleton points d coordinates each."""
        m = self.n_node
        ncand = np.zeros(m, np.int32); so = np.zeros(m + 1, np.int32); uo = np.zeros(m + 1, np.int32)
        lib().ora_h2_bases(self._h, _p(ncand, _i32p), _p(so, _i32p), _p(uo, _i32p))
        U = np.ctypeslib.as_array(lib().ora_h2_U(self._h), shape=(max(int(uo[-1]), 1),)).copy()
        skel = np.ctypeslib.as_array(lib().ora_h2_skel(self._h), shape=(max(int(so[-1]) * self.d, 1),)).copy()
        return ncand, so, uo, U, skel

    def product(self, Y=None, nthreads=None):
        Y = self.Y if Y is None else np.ascontiguousarray(Y, dtype=np.float64)
        s = np.zeros(self.n); v = np.zeros((self.d, self.n))
        lib().ora_h2_product(self._h, _p(Y, _f64p), _p(s, _f64p), _p(v, _f64p),
                             nthreads or nthreads_default())
        return s, v


def proxies(d, h):
    n = lib().ora_h2_n_proxy(d)
    out = np.zeros((d, n))
    lib().ora_h2_proxies(d, float(h), _p(out, _f64p))
    return out


def run(P, Y0, n_iter=1000, learning_rate=None, h2_tol=1e-2, h2_rebuild_freq=3,
        h2_rebuild_freq_early=10, h2_leaf_size=100, use_h2=True, rep_reuse=True, reorder=True,
        early_exag=12.0, early_exag_iter=250, momentum=0.8, initial_momentum=0.5,
        momentum_switch_iter=250, nthreads=None, iter_begin=0, iter_end=0, return_state=False):
    """The whole optimisation phase; returns (Y (d, n) in the caller's order, kl)."""
    Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
    d, n = Y0.shape
    rp = np.ascontiguousarray(P.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(P.indices, dtype=np.int32)
    pv = np.ascontiguousarray(P.data, dtype=np.float64)
    L = lib()
    st = L.ora_state_create(n, d, _p(rp, _i32p), _p(ci, _i32p), _p(pv, _f64p), _p(Y0, _f64p))
    prm = RunParams(n_iter=n_iter, learning_rate=learning_rate or max(n / 12.0, 200.0),
                    momentum=momentum, initial_momentum=initial_momentum,
                    momentum_switch_iter=momentum_switch_iter, early_exag=early_exag,
                    early_exag_iter=early_exag_iter, h2_tol=h2_tol, h2_rebuild_freq=h2_rebuild_freq,
                    h2_rebuild_freq_early=max(h2_rebuild_freq_early, h2_rebuild_freq),
                    h2_leaf_size=h2_leaf_size, use_h2=int(use_h2), rep_reuse=int(rep_reuse),
                    reorder=int(reorder), nthreads=nthreads or nthreads_default(),
                    iter_begin=iter_begin, iter_end=iter_end)
    rc = L.ora_run(st, ctypes.byref(prm))
    if rc != 0:
        L.ora_state_free(st)
        raise RuntimeError("ora_run failed")
    Y = np.zeros((d, n))
    L.ora_get_embedding(st, _p(Y, _f64p))
    kl_val = st.contents.kl
    n_rebuild = st.contents.n_rebuild
    L.ora_state_free(st)
    if return_state:
        return Y, kl_val, n_rebuild
    return Y, kl_val


# ---------------------------------------------------------------------------------------
# The reference's own exact path (oracle/_ref), driven like its Python backend does
# ---------------------------------------------------------------------------------------
def ref_available():
    return _REF_PATH.exists()


_ref = None


class _RefParams(ctypes.Structure):
    """tsne_params_t of the reference header (include/tsne_h2pack.h:27-85), 160 bytes."""
    _fields_ = [
        ("n_iter", ctypes.c_int), ("_pad1", ctypes.c_int), ("perplexity", ctypes.c_double),
        ("learning_rate", ctypes.c_double), ("momentum", ctypes.c_double),
        ("initial_momentum", ctypes.c_double), ("momentum_switch_iter", ctypes.c_int),
        ("_pad2", ctypes.c_int), ("early_exag", ctypes.c_double), ("early_exag_iter", ctypes.c_int),
        ("use_vptree", ctypes.c_int), ("h2_tol", ctypes.c_double), ("h2_rebuild_freq", ctypes.c_int),
        ("h2pack_print_level", ctypes.c_int), ("init_method", ctypes.c_int),
        ("random_seed", ctypes.c_int), ("verbose", ctypes.c_int), ("print_freq", ctypes.c_int),
        ("enable_early_stopping", ctypes.c_int), ("_pad4", ctypes.c_int),
        ("convergence_tol", ctypes.c_double), ("convergence_patience", ctypes.c_int),
        ("min_iter", ctypes.c_int), ("sklearn_compatible", ctypes.c_int),
        ("enable_profiling", ctypes.c_int), ("profiling_output_file", ctypes.c_char_p),
        ("num_threads", ctypes.c_int), ("h2_leaf_size", ctypes.c_int),
        ("h2_rebuild_freq_early", ctypes.c_int), ("_pad5", ctypes.c_int),
        ("init_Y", _f64p),
    ]


class _RefCSR(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_int), ("n_cols", ctypes.c_int), ("nnz", ctypes.c_int),
                ("row_ptr", _i32p), ("col_idx", _i32p), ("values", _f64p)]


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference build missing: {_REF_PATH}")
        os.environ.setdefault("TSNE_H2PACK_NO_PROXY_CACHE", "1")
        L = ctypes.CDLL(str(_REF_PATH))
        L.compute_P_from_knn_distances.argtypes = [_f64p, _i32p, _i32p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_int]
        L.compute_P_from_knn_distances.restype = ctypes.POINTER(_RefCSR)
        L.sparse_matrix_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.sparse_matrix_create.restype = ctypes.POINTER(_RefCSR)
        L.sparse_matrix_destroy.argtypes = [ctypes.POINTER(_RefCSR)]
        L.tsne_init_with_P.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(_RefParams), ctypes.POINTER(_RefCSR)]
        L.tsne_init_with_P.restype = ctypes.c_void_p
        L.tsne_run.argtypes = [ctypes.c_void_p]
        L.tsne_run.restype = ctypes.c_int
        L.tsne_get_embedding.argtypes = [ctypes.c_void_p, _f64p]
        L.tsne_destroy.argtypes = [ctypes.c_void_p]
        L.compute_kl_divergence.argtypes = [ctypes.c_void_p]
        L.compute_kl_divergence.restype = ctypes.c_double
        L.initialize_embedding.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p,
                                           ctypes.c_uint]
        L.shim_h2_assemble.argtypes = ([ctypes.c_int] * 4 + [_i32p, _f64p] + [_i32p] * 6 +
                                       [ctypes.c_int, _i32p, ctypes.c_int, _i32p, _i32p, _i32p, _f64p, _i32p,
                                        _f64p, _i32p])
        L.shim_h2_assemble.restype = ctypes.c_void_p
        L.shim_h2_free.argtypes = [ctypes.c_void_p]
        L.shim_ref_repulsion.argtypes = [ctypes.c_void_p, _f64p, ctypes.c_int, ctypes.c_int, _f64p]
        L.shim_ref_repulsion.restype = ctypes.c_double
        _ref = L
    return _ref


def ref_conditional_P(dist, indices, indptr, perplexity, nthreads=1):
    L = ref_lib()
    dist = np.ascontiguousarray(dist, dtype=np.float64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    indptr = np.ascontiguousarray(indptr, dtype=np.int32)
    n, nnz = len(indptr) - 1, len(dist)
    m = L.compute_P_from_knn_distances(_p(dist, _f64p), _p(indices, _i32p), _p(indptr, _i32p), n,
                                       nnz, ctypes.c_double(perplexity), int(nthreads))
    vals = np.ctypeslib.as_array(m.contents.values, shape=(nnz,)).copy()
    L.sparse_matrix_destroy(m)
    return vals


def ref_init_embedding(n, d, seed):
    Y = np.zeros((d, n))
    ref_lib().initialize_embedding(_p(Y, _f64p), n, d, 0, None, ctypes.c_uint(seed & 0xFFFFFFFF))
    return Y


def ref_run(P, Y0, n_iter, learning_rate=None, early_exag=12.0, early_exag_iter=250,
            sklearn_compatible=1, nthreads=1, attr_f32=0, h2=False, h2_tol=1e-2, h2_rebuild_freq=3,
            h2_rebuild_freq_early=10, h2_leaf_size=100, attr_generic=False, profile=None, timing=None):
    """The reference's own tsne_run; P: symmetric normalised scipy CSR; Y0: (d, n).

    h2=False: its exact-repulsion path (h2_rebuild_freq=999999, i.e. method='exact').
    h2=True: its H2 path, with every H2 matrix built by the oracle behind the H2Pack
    interface (ref_shim/h2_assemble.c): the reference's rebuild schedule, force reuse,
    renumbering, fused product, Z identity and force run on the oracle's matrices.
    attr_generic selects its FP64 attractive pass (TSNE_ATTR_GENERIC=1) instead of the
    2D single-precision gather. profile: a path; the reference writes its per-iteration
    stage times there (tsne_write_profiling_data's CSV), read back by ref_profile_csv.
    timing: a dict that receives 'run_s', the wall time of tsne_run alone (the reference's
    optimisation phase)."""
    L = ref_lib()
    os.environ["TSNE_ATTR_F32"] = str(attr_f32)
    os.environ["TSNE_ATTR_GENERIC"] = "1" if attr_generic else "0"
    Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
    d, n = Y0.shape
    prm = _RefParams(n_iter=n_iter, perplexity=30.0,
                     learning_rate=learning_rate or max(n / 12.0, 200.0), momentum=0.8,
                     initial_momentum=0.5, momentum_switch_iter=250, early_exag=early_exag,
                     early_exag_iter=early_exag_iter, use_vptree=2, h2_tol=h2_tol if h2 else 1e-4,
                     h2_rebuild_freq=h2_rebuild_freq if h2 else 999999, init_method=1, random_seed=0,
                     verbose=0, print_freq=50, convergence_tol=1e-5, convergence_patience=300, min_iter=250,
                     sklearn_compatible=sklearn_compatible, num_threads=nthreads, h2_leaf_size=h2_leaf_size,
                     h2_rebuild_freq_early=h2_rebuild_freq_early if h2 else 999999, init_Y=_p(Y0, _f64p),
                     enable_profiling=1 if profile else 0,
                     profiling_output_file=str(profile).encode() if profile else None)
    nnz = P.nnz
    m = L.sparse_matrix_create(n, n, nnz)
    ctypes.memmove(m.contents.row_ptr, np.ascontiguousarray(P.indptr, np.int32).ctypes.data, 4 * (n + 1))
    ctypes.memmove(m.contents.col_idx, np.ascontiguousarray(P.indices, np.int32).ctypes.data, 4 * nnz)
    ctypes.memmove(m.contents.values, np.ascontiguousarray(P.data, np.float64).ctypes.data, 8 * nnz)
    ws = L.tsne_init_with_P(None, n, 0, d, ctypes.byref(prm), m)
    if not ws:
        raise RuntimeError("reference tsne_init_with_P returned NULL")
    try:
        t0 = time.perf_counter()
        if L.tsne_run(ws) != 0:
            raise RuntimeError("reference tsne_run failed")
        if timing is not None:
            timing["run_s"] = time.perf_counter() - t0
        Y = np.zeros((d, n))
        L.tsne_get_embedding(ws, _p(Y, _f64p))
        kl_val = L.compute_kl_divergence(ws)
    finally:
        L.tsne_destroy(ws)
    return Y, kl_val


def ref_profile_csv(path):
    """Per-iteration stage times (seconds) from the reference's profiling CSV: a dict of
    arrays keyed by its columns (p_matvec = attractive pass, h2_rebuild, h2_matvec_s = fused
    product, z_computation, gradient = update, other)."""
    rows = [ln.strip().split(",") for ln in Path(path).read_text().splitlines()
            if ln and not ln.startswith("#")]
    head, body = rows[0], [r for r in rows[1:] if len(r) == len(rows[0])]
    return {k: np.array([float(r[i]) for r in body]) for i, k in enumerate(head)}


class Runner:
    """A persistent oracle state for timing bounded samples of the optimisation phase."""

    def __init__(self, P, Y0, nthreads=None, **kw):
        Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
        self.d, self.n = Y0.shape
        self._arrays = (np.ascontiguousarray(P.indptr, dtype=np.int32),
                        np.ascontiguousarray(P.indices, dtype=np.int32),
                        np.ascontiguousarray(P.data, dtype=np.float64))
        rp, ci, pv = self._arrays
        self.st = lib().ora_state_create(self.n, self.d, _p(rp, _i32p), _p(ci, _i32p), _p(pv, _f64p),
                                         _p(Y0, _f64p))
        n = self.n
        self.prm = RunParams(n_iter=kw.get("n_iter", 1000), learning_rate=kw.get("learning_rate") or max(n / 12.0, 200.0),
                             momentum=0.8, initial_momentum=0.5, momentum_switch_iter=250,
                             early_exag=12.0, early_exag_iter=250, h2_tol=kw.get("h2_tol", 1e-2),
                             h2_rebuild_freq=kw.get("h2_rebuild_freq", 3),
                             h2_rebuild_freq_early=kw.get("h2_rebuild_freq_early", 10),
                             h2_leaf_size=kw.get("h2_leaf_size", 100), use_h2=1, rep_reuse=1, reorder=1,
                             nthreads=nthreads or nthreads_default(), iter_begin=0, iter_end=0)

    def run(self, begin, end):
        self.prm.iter_begin, self.prm.iter_end = begin, end
        if lib().ora_run(self.st, ctypes.byref(self.prm)) != 0:
            raise RuntimeError("ora_run failed")

    def close(self):
        if self.st:
            lib().ora_state_free(self.st)
            self.st = None

    def __del__(self):
        self.close()


def ref_h2_repulsion(h2, Y=None):
    """The reference's compute_repulsive_forces_h2pack (src/tsne_h2pack.c:389-630, with its
    fused product src/tsne_h2_matmul.c:225-452) run on the H2 matrix `h2` that the oracle
    built: returns (F, Z), F (d, n) in the caller's order."""
    Y = h2.Y if Y is None else np.ascontiguousarray(Y, dtype=np.float64)
    ncand, so, uo, U, skel = h2.bases()
    return ref_h2_repulsion_on(Y, h2.perm(), h2.nodes(), h2.lists(), h2.max_level, h2.ranks(), ncand, U, uo,
                               skel, so)


def ref_h2_repulsion_on(Y, perm, nodes, lists, max_level, rank, ncand, U, U_off, skel, skel_off):
    """The reference's repulsive force on any H2 matrix given as arrays: perm (tree position
    -> point), the node table (dict of start, end, level, first_child, n_child, is_leaf), the
    per-target lists (far_ptr, far_idx, near_ptr, near_idx, both directions of every pair),
    ranks, and the bases packed as by H2.bases(). Returns (F, Z)."""
    L = ref_lib()
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    d, n = Y.shape
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    coord = np.ascontiguousarray(Y[:, perm])
    fp, fi, npt, ni = lists
    n_node = len(rank)
    adm, inadm = [], []
    for t in range(n_node):
        adm += [(t, s) for s in fi[fp[t]:fp[t + 1]] if s > t]
        inadm += [(t, s) for s in ni[npt[t]:npt[t + 1]] if s > t]
    adm = np.ascontiguousarray(np.array(adm, np.int32).reshape(-1, 2))
    inadm = np.ascontiguousarray(np.array(inadm, np.int32).reshape(-1, 2))
    arr = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    keep = [arr(nodes[k]) for k in ("start", "end", "level", "first_child", "n_child", "is_leaf")]
    rank, ncand, U_off, skel_off = arr(rank), arr(ncand), arr(U_off), arr(skel_off)
    U, skel = f64(U), f64(skel)
    h = L.shim_h2_assemble(n, d, int(max_level), n_node, _p(perm, _i32p), _p(coord, _f64p),
                           *[_p(a, _i32p) for a in keep], len(adm), _p(adm, _i32p), len(inadm),
                           _p(inadm, _i32p), _p(rank, _i32p), _p(ncand, _i32p), _p(U, _f64p),
                           _p(U_off, _i32p), _p(skel, _f64p), _p(skel_off, _i32p))
    grad = np.zeros((d, n))
    try:
        Z = L.shim_ref_repulsion(h, _p(Y, _f64p), d, n, _p(grad, _f64p))
    finally:
        L.shim_h2_free(h)
    return -grad, Z
