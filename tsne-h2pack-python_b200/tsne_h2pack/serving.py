"""Batched and served embedding jobs on one GPU (the engine's tsne_server_* entry points).

    >>> from tsne_h2pack.serving import EmbeddingServer
    >>> with EmbeddingServer(max_concurrent=8, hbm_budget_gb=150) as srv:
    ...     jobs = [srv.submit(P, n_components=2, n_iter=750) for P in graphs]
    ...     results = [srv.wait(j) for j in jobs]      # (Y, info) each

Jobs queue in arrival order and start when a slot and device memory are free (continuous
batching); the running jobs' kernels overlap on the GPU, and each job's result is bit for bit
the one it gets alone. `submit` returns at once, so a request loop can keep submitting while
earlier jobs run. This has no counterpart in the reference package, which runs one embedding
per call.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from ._backend import DTYPE, TSNEParams, get_backend, scipy_csr_to_c_sparse_matrix


class JobInfo(ctypes.Structure):
    """tsne_job_info_t (include/tsne_h2pack.h)."""
    _fields_ = [("job", ctypes.c_int), ("status", ctypes.c_int), ("n_point", ctypes.c_int),
                ("low_dim", ctypes.c_int), ("latency_s", ctypes.c_double), ("queue_s", ctypes.c_double),
                ("run_s", ctypes.c_double), ("kl", ctypes.c_double), ("start_s", ctypes.c_double),
                ("end_s", ctypes.c_double)]


@dataclass
class JobResult:
    job: int
    ok: bool
    n_point: int
    low_dim: int
    latency_s: float
    queue_s: float
    run_s: float
    kl: float
    start_s: float
    end_s: float


def _bind(lib):
    if getattr(lib, "_server_bound", False):
        return
    lib.tsne_server_create.argtypes = [ctypes.c_int, ctypes.c_double]
    lib.tsne_server_create.restype = ctypes.c_void_p
    lib.tsne_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TSNEParams),
                                       ctypes.c_void_p]
    lib.tsne_server_submit.restype = ctypes.c_int
    lib.tsne_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(JobInfo)]
    lib.tsne_server_wait.restype = ctypes.c_int
    lib.tsne_server_pending.argtypes = [ctypes.c_void_p]
    lib.tsne_server_pending.restype = ctypes.c_int
    lib.tsne_server_destroy.argtypes = [ctypes.c_void_p]
    lib.tsne_server_destroy.restype = None
    lib.tsne_release_cached_memory.argtypes = []
    lib.tsne_release_cached_memory.restype = ctypes.c_int
    lib._server_bound = True


class EmbeddingServer:
    """Runs embedding jobs concurrently on the current CUDA device.

    max_concurrent: jobs running at once (each a workspace with its own stream).
    hbm_budget_gb: device memory the running jobs may hold, by the engine's upper estimate
    (a job larger than the budget still runs, alone).
    autotune: True (or a LeafTuner) to set each job's h2_leaf_size from the leaf-size autotuner
    of its size bucket (tsne_h2pack.autotune), unless the job sets it itself.
    """

    def __init__(self, max_concurrent=8, hbm_budget_gb=150.0, autotune=False):
        self._tuner = None
        if autotune:
            from .autotune import LeafTuner
            self._tuner = autotune if isinstance(autotune, LeafTuner) else LeafTuner()
        self._be = get_backend()
        self._lib = self._be._lib
        _bind(self._lib)
        self._h = self._lib.tsne_server_create(int(max_concurrent), float(hbm_budget_gb))
        if not self._h:
            raise RuntimeError("tsne_server_create failed (no CUDA device?)")
        self._keep = {}

    def submit(self, P, n_components=2, params=None, **overrides):
        """Queue one job for the joint probability matrix P (scipy CSR, n x n). `params` is a
        TSNEParams (default: create_default_params()); keyword overrides set its fields
        (n_iter, learning_rate, h2_tol, init_Y as an (n_components, n) array, ...). Returns
        the job id."""
        n = P.shape[0]
        p = params if params is not None else self._be.create_default_params()
        init = overrides.pop("init_Y", None)
        for k, v in overrides.items():
            setattr(p, k, v)
        if self._tuner is not None and "h2_leaf_size" not in overrides:
            p.h2_leaf_size = self._tuner.leaf_for(n, n_components, p.h2_tol)
        if init is not None:
            init = np.ascontiguousarray(init, dtype=np.float64)
            if init.shape != (n_components, n):
                raise ValueError(f"init_Y must have shape ({n_components}, {n})")
            p.init_method = 1
            p.init_Y = init.ctypes.data_as(ctypes.POINTER(DTYPE))
        Pc = scipy_csr_to_c_sparse_matrix(P.tocsr(), self._lib)
        job = self._lib.tsne_server_submit(self._h, n, int(n_components), ctypes.byref(p), Pc)
        if job < 0:
            self._lib.sparse_matrix_destroy(Pc)
            raise ValueError("tsne_server_submit rejected the job")
        self._keep[job] = (n, n_components)
        return job

    def wait(self, job):
        """Block until `job` ends; returns (Y (n, n_components) or None, JobResult)."""
        n, d = self._keep.pop(job)
        Y = np.zeros((d, n), dtype=np.float64)
        info = JobInfo()
        rc = self._lib.tsne_server_wait(self._h, int(job), Y.ctypes.data, ctypes.byref(info))
        res = JobResult(job=info.job, ok=(rc == 0), n_point=info.n_point, low_dim=info.low_dim,
                        latency_s=info.latency_s, queue_s=info.queue_s, run_s=info.run_s, kl=info.kl,
                        start_s=info.start_s, end_s=info.end_s)
        return (Y.T.copy() if rc == 0 else None), res

    def pending(self):
        return self._lib.tsne_server_pending(self._h)

    def close(self):
        if self._h:
            self._lib.tsne_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
