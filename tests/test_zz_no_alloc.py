"""tsne_exact_repulsion_static, the entry point for callers that cannot allocate device memory
(a server under a fixed, pre-carved memory budget, code that cannot take an allocation's
implicit device synchronisation, hosts with their own allocator): its scratch is a fixed
__device__ array in the library. Checked through the C ABI on two calls in a row (the second
call must not see the first call's scratch) against

  - the existing exact-repulsion entry point (compute_repulsive_forces_h2pack of a workspace
    without an H2 matrix): F max rel 1e-5, Z rel 1e-6;
  - the FP64 oracle (exact sums and the reference's Z and force formulas in double precision)
    in 2D and 3D, at its largest accepted size (65,536 points) and on a wide embedding
    (coordinates up to 2,000, where the reference's Z identity cancels): F max rel 1e-5,
    Z rel 2e-6.

Collected last, so that a run stopping at its first failure has run everything else."""
import ctypes

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, problem, rel

pytestmark = pytest.mark.gpu

MAX_POINTS = 65536


def _bind(lib):
    lib.tsne_exact_repulsion_static.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p]
    lib.tsne_exact_repulsion_static.restype = ctypes.c_int
    return lib.tsne_exact_repulsion_static


def _static_force(fn, Y):
    """F (d, n) and Z of the no-allocation entry point for Y (d, n), through device buffers."""
    import torch
    d, n = Y.shape
    Yd = torch.tensor(np.ascontiguousarray(Y.T), dtype=torch.float32, device="cuda")
    Fd = torch.full_like(Yd, float("nan"))
    Zd = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert fn(Yd.data_ptr(), n, d, Fd.data_ptr(), Zd.data_ptr(), None) == 0
    torch.cuda.synchronize()
    return Fd.cpu().numpy().T.astype(np.float64), float(Zd.cpu().item())


def _ring_P(n):
    """A symmetric P linking each point to the next (the repulsion does not read P)."""
    i = np.arange(n)
    rows = np.concatenate([i, (i + 1) % n])
    cols = np.concatenate([(i + 1) % n, i])
    return csr_matrix((np.full(2 * n, 0.5 / n), (rows, cols)), shape=(n, n))


@pytest.mark.parametrize("d", [2, 3])
def test_static_scratch_entry_point_matches_exact_path(d):
    X, G, P, _ = problem(1500, seed=2, dim=20)
    n = P.shape[0]
    Y0 = O.init_embedding(n, d, 3)
    eng = Engine(P, Y0, n_iter=1)          # n < 2000: the workspace uses exact sums
    fn = _bind(eng.lib)
    rng = np.random.default_rng(0)
    for call in range(2):
        # two different embeddings, so a call that read the previous call's scratch would fail;
        # narrow enough that the existing entry point's identity (single-precision sums) keeps
        # its digits (the FP64 comparison below covers wide embeddings)
        Y = (Y0 * 1e4 + rng.normal(scale=(1.0 + 2.0 * call), size=Y0.shape)).astype(np.float32).astype(np.float64)
        F_ref, Z_ref = eng.repulsive(Y)
        F, Z = _static_force(fn, Y)
        assert rel(F, F_ref) < 1e-5, call
        assert abs(Z - Z_ref) < 1e-6 * abs(Z_ref), call
    eng.close()


def _fp64(Y):
    s, v = O.exact_sv(Y)
    Z, F = O.z_force(Y, s, v)
    return F, Z


@pytest.mark.parametrize("d,n,width", [(2, MAX_POINTS, 30.0), (3, MAX_POINTS, 30.0), (2, 4000, 2000.0),
                                       (3, 4000, 2000.0)])
def test_static_scratch_entry_point_matches_fp64_oracle(d, n, width):
    """Clusters spread over [-width, width]^d with unit-scale neighbourhoods."""
    from tsne_h2pack._backend import get_backend
    fn = _bind(get_backend()._lib)
    rng = np.random.default_rng(n + d)
    for call in range(2):
        centres = rng.uniform(-width, width, size=(d, 40))
        lab = rng.integers(0, 40, size=n)
        Y = (centres[:, lab] + rng.normal(scale=1.0 + 2.0 * call, size=(d, n))).astype(np.float32).astype(np.float64)
        F_ref, Z_ref = _fp64(Y)
        F, Z = _static_force(fn, Y)
        err_f, err_z = rel(F, F_ref), abs(Z - Z_ref) / Z_ref
        print(f"d={d} n={n} width={width} call {call}: F max rel {err_f:.2e}, Z rel {err_z:.2e}")
        assert err_f < 1e-5, call
        assert err_z < 2e-6, call


def test_static_scratch_entry_point_refusals_and_bad_input():
    import torch
    from tsne_h2pack._backend import get_backend
    fn = _bind(get_backend()._lib)
    n, d = 300, 2
    Y = torch.randn(n, d, dtype=torch.float32, device="cuda")
    F = torch.empty_like(Y)
    Z = torch.zeros(1, dtype=torch.float64, device="cuda")
    # sizes beyond the fixed scratch, and an output written over the input, are refused
    # on the host, before any device work
    assert fn(Y.data_ptr(), MAX_POINTS + 1, d, F.data_ptr(), Z.data_ptr(), None) == -1
    assert fn(Y.data_ptr(), n, d, Y.data_ptr(), Z.data_ptr(), None) == -1
    assert fn(Y.data_ptr(), n, 4, F.data_ptr(), Z.data_ptr(), None) == -1
    # a NaN in Y: Z comes back non-finite and F is zero
    Y[7, 1] = float("nan")
    assert fn(Y.data_ptr(), n, d, F.data_ptr(), Z.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert not np.isfinite(Z.item())
    assert torch.count_nonzero(F).item() == 0
