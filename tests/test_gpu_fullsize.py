"""The device H2 repulsion at the benchmark sizes, against full-N FP64 sums.

Workloads (the benchmark's mixture recipe, exact k = 90 graph built on the GPU, perplexity 30,
init='random'):
  - 1,000,000 points, 2D, seed 1, h2_tol 1e-2 (the headline configuration);
  - 500,000 points, 3D, seed 2, h2_tol 3e-2.

At rebuild iterations spread over the 1000-iteration run (the first build, the first
renumbering at 30, the late schedule at 300 and the last iteration), the repulsive force that
the device computed at that rebuild, and its Z, are compared with exact sums over all N points
in double precision:
  - force: on a seeded random subset of 50,000 rows, the oracle's exact FP64 sums over all N
    points (oracle.exact_rows, the reference's s, v and force formulas) with the exact Z;
    relative 2-norm error over the subset <= h2_tol;
  - Z: |Z_device - Z_exact| / Z_exact <= h2_tol, with Z_exact the FP64 sum of
    (1 + r^2)^-1 over all N^2 - N pairs (helpers.exact_Z_torch, itself checked against the
    oracle's exact Z at 20,000 points to 1e-10).
"""
import numpy as np
import pytest

import oracle as O
from helpers import Engine, exact_Z_torch, rel2

pytestmark = pytest.mark.gpu

CHECK_ITERS = (0, 30, 300, 999)
SUBSET = 50_000


def _workload(n, seed):
    from tsne_h2pack._backend import get_backend
    from tsne_h2pack._synthetic import knn_graph_torch, mixture_zipf
    X, _ = mixture_zipf(n, seed=seed)
    G = knn_graph_torch(X, 90, chunk=4096)
    return get_backend().joint_P(G, 30.0)


def test_exact_Z_checker_matches_oracle():
    rng = np.random.default_rng(5)
    for d in (2, 3):
        Y = rng.normal(scale=20.0, size=(d, 20_000))
        s, v = O.exact_sv(Y)
        Zo, _ = O.z_force(Y, s, v)
        assert abs(exact_Z_torch(Y) - Zo) <= 1e-10 * Zo


def _check_run(P, d, seed, h2_tol):
    n = P.shape[0]
    Y0 = O.init_embedding(n, d, seed)
    eng = Engine(P, Y0, n_iter=1000, h2_tol=h2_tol)
    rows = np.sort(np.random.default_rng(12345).choice(n, SUBSET, replace=False)).astype(np.int32)
    done, out = 0, []
    for it in CHECK_ITERS:
        if it > done:
            eng.run(done, it)
        Y, _, _ = eng.state()                 # the embedding at the start of iteration `it`
        eng.run(it, it + 1)                   # `it` is a rebuild iteration: its force is stored
        done = it + 1
        _, F, Z = eng.state()
        s, v = O.exact_rows(Y, rows)
        Ze = exact_Z_torch(Y)
        Fe = (4.0 / Ze) * (Y[:, rows] * s[None, :] - v)
        ferr, zerr = rel2(F[:, rows], Fe), abs(Z - Ze) / Ze
        out.append((it, ferr, zerr))
        print(f"n={n} d={d} iteration {it}: force rel {ferr:.3e}, Z rel {zerr:.3e} (h2_tol {h2_tol:g})")
    eng.close()
    for it, ferr, zerr in out:
        assert ferr <= h2_tol, (it, ferr)
        assert zerr <= h2_tol, (it, zerr)


def test_h2_force_at_1M_points_2d():
    _check_run(_workload(1_000_000, 1), 2, 1, 1e-2)


def test_h2_force_at_500K_points_3d():
    _check_run(_workload(500_000, 2), 3, 2, 3e-2)
