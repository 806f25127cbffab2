"""bench.py's reference arm on the CPU: one JSON line with the contract's keys, from a small
cached workload (the graph cache stands in for the GPU-built k-NN graph)."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

from helpers import problem

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line(tmp_path):
    n = 3000
    X, G, P, _ = problem(n, seed=2, dim=20)
    G, P = G.tocsr(), P.tocsr()
    cache = tmp_path / "g.npz"
    np.savez(cache, gd=G.data, gi=G.indices, gp=G.indptr, pd=P.data, pi=P.indices, pp=P.indptr)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--n", str(n),
                        "--graph-cache", str(cache), "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in out, k
    assert out["impl"] == "reference" and out["unit"] == "s" and out["higher_is_better"] is False
    assert out["value"] > 0 and out["e2e"]["value"] == out["value"]
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["e2e"]["d2h_bytes_per_step"] == 0
    cb = out["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == out["value"]
    assert cb["sample"]
    assert out["steps"] >= 1 and "steps_requested" in out and cb["split_s"]["h2_rebuild"] >= 0


def test_parity_scores_on_the_cpu():
    """bench.parity: an embedding against itself passes with zero differences; against a
    scrambled copy it fails (the scores see the neighbourhoods)."""
    sys.path.insert(0, str(ROOT))
    import bench
    import oracle as O
    n = 3000
    X, G, P, _ = problem(n, seed=2, dim=20)
    Y, kl = O.run(P.tocsr(), O.init_embedding(n, 2, 1), n_iter=300)
    out = bench.parity(G.tocsr(), P.tocsr(), Y, kl, Y, kl)
    assert out["pass"] and out["knn30_preservation"]["diff_points"] == 0 and out["kl_run"]["rel_diff"] == 0
    assert out["knn10_preservation"]["ours"] > 0.1
    Ys = Y[:, np.random.default_rng(0).permutation(n)]
    bad = bench.parity(G.tocsr(), P.tocsr(), Ys, kl, Y, kl)
    assert not bad["pass"] and bad["knn30_preservation"]["diff_points"] < -5
