"""Batched and served jobs (tsne_server_* through tsne_h2pack.serving) on the GPU.

Each job is an independent workspace with its own stream; its result must be bit for bit the
one the plain path (tsne_init_with_P + tsne_run) gives for the same input, whatever runs
beside it. Admission: a job starts only when it fits under the HBM budget next to the running
ones (or runs alone), and a job submitted while others run starts before they end when a slot
is free.
"""
import time

import numpy as np
import pytest

import oracle as O
from helpers import Engine, problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jobs():
    out = []
    for n, d, seed, perp, clusters in ((2500, 2, 1, 30.0, 6), (3000, 3, 2, 10.0, 4), (1500, 2, 3, 30.0, 5),
                                       (4000, 2, 4, 50.0, 8)):
        X, G, P, _ = problem(n, seed=seed, k=min(90, int(3 * perp)), perplexity=perp, dim=20, n_clusters=clusters)
        out.append((P, O.init_embedding(n, d, seed + 10)))
    return out


def _alone(P, Y0, n_iter):
    eng = Engine(P, Y0, n_iter=n_iter)
    eng.run_all()
    Y, kl = eng.embedding(), eng.kl()
    eng.close()
    return Y, kl


def _submit(srv, P, Y0, n_iter):
    d, n = Y0.shape
    # the parameters Engine uses
    return srv.submit(P, n_components=d, init_Y=Y0, n_iter=n_iter, verbose=0,
                      learning_rate=max(n / 12.0, 200.0), h2_tol=1e-2, h2_rebuild_freq=3,
                      h2_rebuild_freq_early=10, h2_leaf_size=100)


def test_batch_results_equal_alone(jobs):
    from tsne_h2pack.serving import EmbeddingServer
    n_iter = 60
    ref = [_alone(P, Y0, n_iter) for P, Y0 in jobs]
    with EmbeddingServer(max_concurrent=4, hbm_budget_gb=100.0) as srv:
        ids = [_submit(srv, P, Y0, n_iter) for P, Y0 in jobs]
        res = [srv.wait(j) for j in ids]
        # a collected result is released: a second wait reports the job but returns -1
        import ctypes
        from tsne_h2pack.serving import JobInfo
        info = JobInfo()
        assert srv._lib.tsne_server_wait(srv._h, ids[0], None, ctypes.byref(info)) == -1
        assert info.status == 0 and info.n_point == jobs[0][0].shape[0]
    assert srv._lib.tsne_release_cached_memory() == 0
    for (Yr, klr), (Y, info) in zip(ref, res):
        assert info.ok
        np.testing.assert_array_equal(Y.T, Yr)
        assert info.kl == klr
    starts = sorted(r.start_s for _, r in res)
    ends = sorted(r.end_s for _, r in res)
    assert starts[1] < ends[0], "four slots and a large budget: jobs must overlap"


def test_budget_admits_one_job_at_a_time(jobs):
    from tsne_h2pack.serving import EmbeddingServer
    with EmbeddingServer(max_concurrent=3, hbm_budget_gb=0.001) as srv:
        ids = [_submit(srv, P, Y0, 20) for P, Y0 in jobs[:3]]
        res = sorted((srv.wait(j)[1] for j in ids), key=lambda r: r.start_s)
    assert all(r.ok for r in res)
    for a, b in zip(res, res[1:]):
        assert b.start_s >= a.end_s, "a job above the budget runs alone"


def test_job_submitted_while_running_starts_early(jobs):
    """Continuous batching: a second request arriving while the first runs is admitted at once
    (a free slot, memory to spare) and its result is still the one it gets alone."""
    from tsne_h2pack.serving import EmbeddingServer
    (P1, Y1), (P2, Y2) = jobs[3], jobs[0]
    ref2 = _alone(P2, Y2, 40)
    with EmbeddingServer(max_concurrent=2, hbm_budget_gb=100.0) as srv:
        a = _submit(srv, P1, Y1, 600)
        time.sleep(0.05)
        b = _submit(srv, P2, Y2, 40)
        Yb, rb = srv.wait(b)
        Ya, ra = srv.wait(a)
    assert ra.ok and rb.ok
    assert rb.start_s < ra.end_s
    np.testing.assert_array_equal(Yb.T, ref2[0])


def test_leaf_autotuner_picks_a_candidate_and_keeps_quality():
    """The leaf-size autotuner measures every candidate on the device, picks the fastest, and
    a job run with its choice keeps the KL of the default leaf size within 1%."""
    import numpy as np
    import oracle as O
    from helpers import Engine, problem
    from tsne_h2pack.autotune import CANDIDATES, LeafTuner
    tuner = LeafTuner()
    leaf = tuner.leaf_for(20000, 2)
    key = (2, 14)
    assert leaf in CANDIDATES and set(tuner.timings[key]) == set(CANDIDATES)
    assert all(t > 0 for t in tuner.timings[key].values())
    assert tuner.leaf_for(30000, 2) == leaf            # same bucket: cached, not re-measured
    X, G, P, _ = problem(20000, seed=9, dim=20)
    Y0 = O.init_embedding(P.shape[0], 2, 4)
    kl = {}
    for lf in (100, leaf):
        eng = Engine(P, Y0, n_iter=300, h2_leaf_size=lf)
        eng.run_all()
        kl[lf] = eng.kl()
        eng.close()
    assert abs(kl[leaf] - kl[100]) <= 0.01 * kl[100], kl
