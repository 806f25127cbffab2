"""The attractive step's forms with more loads in flight (TSNE_ATTR_PIPE) against the default:

  - 1: each lane loads its next 4 entries of the row before the current gathers;
  - 2: two rows per half-warp (k_attr_pair);
  - 3: each lane loads its next 4 columns before the current gathers;
  - 4: the same across the rows of a half-warp (k_attr_stream).

Both keep every row's sums over the same lanes in the same order, so a run equals the default
run through iteration 32 (past the renumbering at 30) to rel 1e-6 (only the centring mean's
FP64 summation order differs, through the grid size), its KL after 200 iterations within 1e-3,
and a form repeated gives the same bits. Also on a ragged P (isolated points, a 3000-entry hub
row and rows of very different lengths paired in one half-warp).
"""
import numpy as np
import pytest

import oracle as O
from helpers import Engine, problem, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mid():
    return problem(20001, seed=5, n_clusters=12, dim=20)


def _run(P, Y0, iters, pipe, monkeypatch):
    monkeypatch.setenv("TSNE_ATTR_PIPE", str(pipe))
    eng = Engine(P, Y0, n_iter=200)
    eng.run(0, iters)
    Y = eng.embedding()
    kl = eng.kl() if iters >= 200 else None
    eng.close()
    return Y, kl


@pytest.mark.parametrize("kind", ["plain", "ragged"])
@pytest.mark.parametrize("pipe", [1, 2, 3, 4])
def test_pipe_forms_equal_default(mid, kind, pipe, monkeypatch):
    X, G, P, _ = mid
    if kind == "ragged":
        from test_gpu_edges import _ragged
        from test_gpu_tiles import _wide_tile
        P = _wide_tile(_ragged(P))
    Y0 = O.init_embedding(P.shape[0], 2, 3)
    Ya, _ = _run(P, Y0, 32, 0, monkeypatch)
    Yb, _ = _run(P, Y0, 32, pipe, monkeypatch)
    Yc, _ = _run(P, Y0, 32, pipe, monkeypatch)
    np.testing.assert_array_equal(Yb, Yc)
    assert rel(Yb, Ya) <= 1e-6
    _, kla = _run(P, Y0, 200, 0, monkeypatch)
    _, klb = _run(P, Y0, 200, pipe, monkeypatch)
    print(f"{kind} pipe {pipe}: KL default {kla:.6f} form {klb:.6f}")
    assert abs(klb - kla) <= 1e-3 * abs(kla)
