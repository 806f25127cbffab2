#!/usr/bin/env python
"""Generate the golden vectors of tests/golden/ from the reference's own code.

The reference's C sources (src/tsne_utils.c, src/tsne_h2pack.c, ...) are compiled unmodified
into oracle/_ref/libtsne_ref.so by `make -C oracle ref`. The fixtures use 400 points and
method='exact' (h2_rebuild_freq 999999), so tsne_run takes the reference's exact-repulsion
branch (src/tsne_h2pack.c:404-491) and no H2 matrix is involved. This script drives that
library the way the reference's Python backend does and stores its outputs:

  init_*      initialize_embedding (src/tsne_utils.c:1111-1150), glibc srand / Box-Muller
  cond_P      compute_P_from_knn_distances (src/tsne_utils.c:952-1105) on a stored k-NN graph
  Y_<it>, kl_<it>
              tsne_run (src/tsne_h2pack.c:1652-2102) on the exact path from a stored Y0, for
              `it` iterations, then compute_kl_divergence

Inputs (the k-NN graph and Y0) are stored beside the outputs, so the tests need neither the
reference nor the generator's random streams. Run from the repository root:

    make -C oracle ref REF_SRC=<reference checkout>/src
    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np
from scipy.sparse import csr_matrix

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tsne-h2pack-python_b200"))

import oracle as O  # noqa: E402
from tsne_h2pack._synthetic import knn_graph, mixture_equal, symmetric_P  # noqa: E402

OUT = Path(__file__).resolve().parent

# problem of the exact-path fixtures: 400 points, 8 dims, 4 clusters, k = 24, perplexity 8
N, DIM, CLUSTERS, K, PERPLEXITY, SEED = 400, 8, 4, 24, 8.0, 3
ITERS_2D = (1, 5, 10, 20)
ITERS_3D = (1, 5, 10)
INIT_CASES = ((1000, 2, 42), (777, 3, 0), (5, 2, 123456))


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libtsne_ref.so is missing: run `make -C oracle ref REF_SRC=...` first")
    out = {}
    for n, d, seed in INIT_CASES:
        out[f"init_{n}_{d}_{seed}"] = O.ref_init_embedding(n, d, seed)

    X, _ = mixture_equal(N, n_clusters=CLUSTERS, dim=DIM, seed=SEED)
    G = knn_graph(X, K)
    G.sort_indices()
    out["g_data"] = G.data.astype(np.float64)
    out["g_indices"] = G.indices.astype(np.int32)
    out["g_indptr"] = G.indptr.astype(np.int32)
    out["perplexity"] = np.float64(PERPLEXITY)
    cond = O.ref_conditional_P(G.data, G.indices, G.indptr, PERPLEXITY)
    out["cond_P"] = cond
    P = symmetric_P(csr_matrix((cond, G.indices, G.indptr), shape=G.shape))

    for d, its, seed in ((2, ITERS_2D, 7), (3, ITERS_3D, 8)):
        Y0 = O.ref_init_embedding(N, d, seed)
        out[f"Y0_{d}d"] = Y0
        for it in its:
            Y, kl = O.ref_run(P, Y0, it, learning_rate=200.0)
            out[f"Y_{d}d_{it}"] = Y
            out[f"kl_{d}d_{it}"] = np.float64(kl)
    np.savez_compressed(OUT / "ref_exact_path.npz", **out)
    print(f"wrote {OUT / 'ref_exact_path.npz'}: {len(out)} arrays")


if __name__ == "__main__":
    main()
