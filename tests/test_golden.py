"""The oracle and the engine against golden vectors of the reference's own code.

tests/golden/ref_exact_path.npz holds outputs of the reference's C sources compiled unmodified
(initialize_embedding, compute_P_from_knn_distances, tsne_run on its exact-repulsion path and
compute_kl_divergence; generator: tests/golden/make_golden.py). The reference is built with
-ffast-math, the oracle without, so the oracle agrees to rounding (FP64 against FP64); the
engine's device state is FP32 and its rounding grows ~2x per iteration like any t-SNE
perturbation, so its trajectory is compared over the first iterations only.

Tolerances:
  - oracle: init rtol 1e-11, conditional P rtol 1e-12, trajectory max rel 1e-12 through 10
    iterations and 1e-8 at 20, KL rel 1e-12
  - engine (host init) bit-identical to the oracle, so rtol 1e-11 against the reference
  - engine (device): conditional P rtol 1e-10; embedding max rel 1e-5 after 1 iteration and
    1e-4 after 5; KL within 0.1% after 10 iterations and 1% after 20
"""
from pathlib import Path

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import oracle as O
from helpers import Engine, rel
from tsne_h2pack._synthetic import symmetric_P

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_exact_path.npz"


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLDEN)
    g = {k: z[k] for k in z.files}
    n = len(g["g_indptr"]) - 1
    g["n"] = n
    g["G"] = csr_matrix((g["g_data"], g["g_indices"], g["g_indptr"]), shape=(n, n))
    g["P"] = symmetric_P(csr_matrix((g["cond_P"], g["g_indices"], g["g_indptr"]), shape=(n, n)))
    return g


def _iters(gold, d):
    return sorted(int(k.split("_")[-1]) for k in gold if k.startswith(f"Y_{d}d_"))


def _init_cases(gold):
    return [tuple(int(x) for x in k.split("_")[1:]) for k in gold if k.startswith("init_")]


def test_fixture_is_complete(gold):
    assert _iters(gold, 2) == [1, 5, 10, 20]
    assert _iters(gold, 3) == [1, 5, 10]
    assert len(_init_cases(gold)) == 3
    assert gold["cond_P"].shape == gold["g_data"].shape


def test_oracle_init_matches_golden(gold):
    for n, d, seed in _init_cases(gold):
        np.testing.assert_allclose(O.init_embedding(n, d, seed), gold[f"init_{n}_{d}_{seed}"], rtol=1e-11, atol=0)


def test_engine_host_init_matches_golden(gold):
    import ctypes
    from tsne_h2pack._backend import get_backend
    lib = get_backend()._lib
    lib.initialize_embedding.argtypes = [np.ctypeslib.ndpointer(np.float64), ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_uint]
    for n, d, seed in _init_cases(gold):
        Y = np.zeros((d, n))
        lib.initialize_embedding(Y, n, d, 0, None, seed)
        np.testing.assert_allclose(Y, gold[f"init_{n}_{d}_{seed}"], rtol=1e-11, atol=0)


def test_oracle_conditional_P_matches_golden(gold):
    c = O.conditional_P(gold["g_data"], gold["g_indptr"], float(gold["perplexity"]))
    np.testing.assert_allclose(c, gold["cond_P"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("d", [2, 3])
def test_oracle_exact_trajectory_matches_golden(gold, d):
    for it in _iters(gold, d):
        Y, kl = O.run(gold["P"], gold[f"Y0_{d}d"], n_iter=it, learning_rate=200.0, use_h2=False)
        assert rel(Y, gold[f"Y_{d}d_{it}"]) < (1e-12 if it <= 10 else 1e-8), (d, it)
        assert abs(kl - gold[f"kl_{d}d_{it}"]) < 1e-12 * abs(gold[f"kl_{d}d_{it}"]), (d, it)


@pytest.mark.gpu
def test_engine_conditional_P_matches_golden(gold):
    from tsne_h2pack._backend import get_backend
    Pc = get_backend().conditional_P(gold["G"], float(gold["perplexity"]))
    np.testing.assert_allclose(Pc.data, gold["cond_P"], rtol=1e-10, atol=1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("d", [2, 3])
def test_engine_exact_path_matches_golden(gold, d):
    for it in _iters(gold, d):
        eng = Engine(gold["P"], gold[f"Y0_{d}d"], n_iter=it, learning_rate=200.0)
        eng.run_all()
        Y, kl = eng.embedding(), eng.kl()
        eng.close()
        if it <= 5:
            assert rel(Y, gold[f"Y_{d}d_{it}"]) < (1e-5 if it == 1 else 1e-4), (d, it)
        assert abs(kl - gold[f"kl_{d}d_{it}"]) < (1e-3 if it <= 10 else 1e-2) * abs(gold[f"kl_{d}d_{it}"]), (d, it)
