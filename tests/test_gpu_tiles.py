"""The shared-column tile form of the 2D attractive pass (attr_tiles.cu) against the CSR pass
it replaces after the renumberings:

  - the tile kernel keeps the CSR kernel's per-row arithmetic, so a run that switches to tiles
    at iteration 30 equals the CSR run through iteration 31 to rel 1e-6 (only the centring
    mean's FP64 summation order differs), and its KL after 200 iterations within 1e-3;
  - the same on a ragged P: isolated points, a 3000-entry hub row and a tile with more
    distinct columns than the shared-memory stage holds (read from global memory);
  - n not a multiple of the tile (64 and 32 rows).
"""
import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, problem, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mid():
    return problem(20001, seed=5, n_clusters=12, dim=20)


def _wide_tile(P, seed=1):
    """P plus 200 random far partners for each of rows 64 .. 127 (one tile whose distinct
    columns exceed the shared-memory stage), symmetric, normalised."""
    rng = np.random.default_rng(seed)
    n = P.shape[0]
    A = P.tocoo()
    r = np.repeat(np.arange(64, 128), 200)
    c = rng.integers(0, n, size=r.size)
    c = np.where(c == r, (c + 1) % n, c)
    w = np.full(r.size, A.data.mean())
    Q = csr_matrix((np.concatenate([A.data, w, w]), (np.concatenate([A.row, r, c]), np.concatenate([A.col, c, r]))),
                   shape=(n, n))
    Q.sum_duplicates()
    Q.sort_indices()
    Q.data /= Q.data.sum()
    return Q


def _run(P, Y0, iters, tiles, monkeypatch, kind_rows=64):
    monkeypatch.setenv("TSNE_ATTR_TILES", "1" if tiles else "0")
    monkeypatch.setenv("TSNE_ATTR_PIPE", "0")   # the CSR form the tile form pairs with
    monkeypatch.setenv("TSNE_ATTR_TILES_FROM", "30")
    monkeypatch.setenv("TSNE_ATTR_TILE_ROWS", "32" if kind_rows == 32 else "64")
    eng = Engine(P, Y0, n_iter=200)
    eng.run(0, iters)
    Y = eng.embedding() if iters < 200 else None
    if iters >= 200:
        Y, kl = eng.embedding(), eng.kl()
    else:
        kl = None
    eng.close()
    return Y, kl


@pytest.mark.parametrize("kind,rows", [("plain", 64), ("ragged", 64), ("plain", 32)])
def test_tiles_equal_csr_pass(mid, kind, rows, monkeypatch):
    X, G, P, _ = mid
    if kind == "ragged":
        from test_gpu_edges import _ragged
        P = _wide_tile(_ragged(P))
    Y0 = O.init_embedding(P.shape[0], 2, 3)
    Ya, _ = _run(P, Y0, 32, False, monkeypatch, rows)
    Yb, _ = _run(P, Y0, 32, True, monkeypatch, rows)
    assert rel(Yb, Ya) <= 1e-6
    Ya, kla = _run(P, Y0, 200, False, monkeypatch, rows)
    Yb, klb = _run(P, Y0, 200, True, monkeypatch, rows)
    print(f"{kind}: KL csr {kla:.6f} tiles {klb:.6f}")
    assert abs(klb - kla) <= 1e-3 * abs(kla)
