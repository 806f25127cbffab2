"""tsne_exact_repulsion_static, the entry point for callers that cannot allocate device memory
(its scratch is a fixed __device__ array in the library), checked through the C ABI against
the existing exact-repulsion entry point (compute_repulsive_forces_h2pack with no H2 matrix)
on two calls in a row. Collected last so that a run stopping at its first failure has run
everything else."""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import Engine, problem, rel

pytestmark = pytest.mark.gpu


def _reference_force(eng, Y):
    """F (d, n) and Z from the existing entry point (exact O(N^2) sums, engine workspace)."""
    F, Z = eng.repulsive(Y)
    return F, Z


def test_static_scratch_entry_point_matches_exact_path():
    import torch
    X, G, P, _ = problem(1500, seed=2, dim=20)
    n, d = P.shape[0], 2
    Y0 = O.init_embedding(n, d, 3)
    eng = Engine(P, Y0, n_iter=1)          # n < 2000: the workspace uses exact sums
    lib = eng.lib
    lib.tsne_exact_repulsion_static.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p]
    lib.tsne_exact_repulsion_static.restype = ctypes.c_int
    rng = np.random.default_rng(0)
    for call in range(2):
        # two different embeddings, so a call that read the previous call's scratch would fail
        Y = (Y0 * 1e4 + rng.normal(scale=(3.0 + 20.0 * call), size=Y0.shape)).astype(np.float32).astype(np.float64)
        F_ref, Z_ref = _reference_force(eng, Y)
        Yd = torch.tensor(np.ascontiguousarray(Y.T), dtype=torch.float32, device="cuda")
        Fd = torch.empty_like(Yd)
        Zd = torch.empty(1, dtype=torch.float64, device="cuda")
        rc = lib.tsne_exact_repulsion_static(Yd.data_ptr(), n, d, Fd.data_ptr(), Zd.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        F = Fd.cpu().numpy().T.astype(np.float64)
        Z = float(Zd.cpu().item())
        assert rel(F, F_ref) < 1e-5, call
        assert abs(Z - Z_ref) < 1e-6 * abs(Z_ref), call
    # sizes beyond the fixed scratch are refused, without touching the device
    assert lib.tsne_exact_repulsion_static(Yd.data_ptr(), 65537, d, Fd.data_ptr(), Zd.data_ptr(), None) == -1
    eng.close()
