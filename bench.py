#!/usr/bin/env python
"""Benchmark of the t-SNE optimisation phase (the reference's "Total optimization time").

Workload: 1,000,000 x 50 float32 Gaussian mixture (100 clusters, Zipf(1.1) sizes, centres
~N(0, 3^2 I), per-dimension std ~U(0.5, 2)), seed 1; exact k = 90 neighbour graph built once
outside timing; perplexity 30; 2D; 1000 iterations (250 at exaggeration 12); h2_tol 1e-2,
rebuild every 3 iterations (10 during early exaggeration), 100 points per leaf;
init='random'. A step is one whole optimisation phase (tsne_run) on that input.

  value   device time of tsne_run (CUDA events on the engine's stream), seconds, max over ranks
  e2e     the same phase through the C ABI with host buffers: sparse_matrix_create + copy of P,
          tsne_init_with_P (upload of P and Y0, first H2 build), tsne_run, tsne_get_embedding,
          compute_kl_divergence, tsne_destroy
  roofline  the attractive pass fused with the update (the kernel launched every iteration)
  cpu_baseline  one whole run of the reference's own tsne_run (compiled from its sources in
          oracle/_ref) on all host cores, on the same P and init, with the reference's own
          per-stage profile; H2Pack's partition and bases, which are absent, are the oracle's
          restatement behind the H2Pack interface (kind "reference"). Without oracle/_ref, a
          bounded sample of the oracle port, extrapolated (kind "port").
  parity_vs_reference  the final embeddings of that run and of the engine's last step scored
          as the reference scores quality (benchmarks/quality.py): in-run KL, common-P KL,
          10-NN and 30-NN preservation, with the pass criterion (KL within 1%, 30-NN within
          0.5 points).

--impl reference times whole runs of that same CPU path as its own line (steps = runs timed).
Multi-GPU (torchrun): every rank runs its own replica of the workload (no collective on the
data path); value is the slowest rank's time.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "tsne-h2pack-python_b200"))

METRIC = "opt-phase s at 1M pts 2D"


def metric_name(n, iters, d=2):
    """The headline metric for the default workload; other sizes name their own."""
    if (n, iters, d) == (1_000_000, 1000, 2):
        return METRIC
    return f"opt-phase s at {n:,} pts {d}D" + ("" if iters == 1000 else f", {iters} iterations")


def data_desc(n, seed=1):
    return f"synthetic: {n:,} x 50 float32 Zipf(1.1) Gaussian mixture, seed {seed}; exact k=90 graph"
PEAKS = ROOT / "MEASURED_PEAKS.json"
# ncu summaries of the roofline kernel on a smaller case (the default 2D form first); the DRAM
# traffic per algorithmic byte scales the traffic to this workload's launch
TRAFFIC = [ROOT / "profiles" / "k_attr_update_pf_200k_full.md", ROOT / "profiles" / "k_attr_update_200k_full.md"]

# the attractive step's form (TSNE_ATTR_PIPE; default 3 in 2D, 0 in 3D), as the engine picks it
ATTR_FORMS = {0: "k_attr_update", 1: "k_attr_update_pf<1> (next step's entries loaded ahead)",
              2: "k_attr_pair (two rows per half-warp)", 3: "k_attr_update_pf<2> (next step's columns loaded ahead)"}


def attr_form(d):
    v = os.environ.get("TSNE_ATTR_PIPE", "")
    if v == "":
        return 3 if d == 2 else 0
    return int(v) if v.isdigit() and int(v) in ATTR_FORMS else 0


def traffic_ratio():
    """DRAM bytes (read + write) per algorithmic byte of the attractive step, from the first
    committed ncu summary present (line 'traffic_over_algorithmic: X'), or None."""
    path = next((p for p in TRAFFIC if p.exists()), None)
    if path is None:
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith("traffic_over_algorithmic:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except (ValueError, IndexError):
                return None
    return None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--dim", type=int, default=2, choices=[2, 3], help="embedding dimension (plain workload)")
    ap.add_argument("--h2-tol", type=float, default=None, help="default 1e-2 in 2D, 3e-2 in 3D")
    ap.add_argument("--seed", type=int, default=None, help="mixture seed: default 1 in 2D, 2 in 3D")
    ap.add_argument("--iters", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-runs", type=int, default=1, help="reference arm: whole runs timed")
    ap.add_argument("--save-embedding", default=None)
    ap.add_argument("--graph-cache", default=None, help="npz file holding the k-NN graph and P")
    ap.add_argument("--profile-csv", default=None, help="write the per-iteration stage CSV of the last step")
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "served", "fit"],
                    help="plain: the 1M-point run (default); batched: many small embeddings through the "
                         "job server; served: Poisson arrivals of embedding jobs; fit: the whole "
                         "TSNE.fit_transform(X) (device k-NN, device P, optimisation)")
    ap.add_argument("--jobs", type=int, default=256, help="batched: number of embeddings")
    ap.add_argument("--rate", type=float, default=2.0, help="served: arrival rate, jobs/s")
    ap.add_argument("--duration", type=float, default=60.0, help="served: arrival window, seconds")
    ap.add_argument("--max-concurrent", type=int, default=16)
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--autotune", action="store_true",
                    help="batched/served: each job's leaf size from the leaf-size autotuner of its size bucket")
    args = ap.parse_args()
    if args.h2_tol is None:
        args.h2_tol = 1e-2 if args.dim == 2 else 3e-2
    if args.seed is None:
        args.seed = 1 if args.dim == 2 else 2
    return args


def workload(n, seed=1, device=0, cache=None):
    """X, graph G (CSR distances) and joint P of the benchmark input (setup, untimed). With
    `cache`, G and P are stored there on the first call and loaded afterwards (so that a
    profiler run sees no setup kernels)."""
    from scipy.sparse import csr_matrix
    from tsne_h2pack._synthetic import knn_graph_torch, mixture_zipf
    from tsne_h2pack._backend import get_backend
    X, _ = mixture_zipf(n, seed=seed)
    if cache and Path(cache).exists():
        z = np.load(cache)
        G = csr_matrix((z["gd"], z["gi"], z["gp"]), shape=(n, n))
        P = csr_matrix((z["pd"], z["pi"], z["pp"]), shape=(n, n))
        return X, G, P
    G = knn_graph_torch(X, 90, device=f"cuda:{device}", chunk=4096 if n > 200_000 else 8192)
    P = get_backend().joint_P(G, 30.0)
    if cache:
        np.savez(cache, gd=G.data, gi=G.indices, gp=G.indptr, pd=P.data, pi=P.indices, pp=P.indptr)
    return X, G, P


def params_for(be, n, iters, h2_tol=1e-2):
    p = be.create_default_params()
    p.n_iter = iters
    p.verbose = 0
    p.perplexity = 30.0
    p.learning_rate = max(n / 12.0, 200.0)
    p.h2_tol, p.h2_rebuild_freq, p.h2_rebuild_freq_early, p.h2_leaf_size = h2_tol, 3, 10, 100
    p.random_seed = 1
    p.init_method = 0
    return p


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        import tempfile
        self.path = Path(tempfile.gettempdir()) / f"tsne_bench_clocks_{os.getpid()}_{index}.csv"
        self.proc = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1])); mx = max(mx, float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        try:
            self.path.unlink()
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def ours(args, rank, world, local):
    import torch
    from tsne_h2pack._backend import TSNEWorkspace, get_backend, scipy_csr_to_c_sparse_matrix
    torch.cuda.set_device(local)
    os.environ["TSNE_KERNEL_TIMING"] = "1"
    be = get_backend()
    lib = be._lib
    lib.tsne_get_timing.argtypes = [ctypes.POINTER(TSNEWorkspace), ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    n, d = args.n, args.dim
    t0 = time.time()
    X, G, P = workload(n, seed=args.seed, device=local, cache=args.graph_cache)
    setup_s = time.time() - t0
    nnz = P.nnz
    Yout = np.zeros((d, n))

    def step():
        """One e2e step through the C ABI; returns (wall s, device run s, attr ms, attr launches, launches)."""
        prm = params_for(be, n, args.iters, args.h2_tol)
        if args.profile_csv:
            prm.enable_profiling = 1
            prm.profiling_output_file = args.profile_csv.encode()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        Pc = scipy_csr_to_c_sparse_matrix(P, lib)
        w1 = time.perf_counter()
        ws = lib.tsne_init_with_P(None, n, 0, d, ctypes.byref(prm), Pc)
        if not ws:
            raise RuntimeError("tsne_init_with_P returned NULL")
        w2 = time.perf_counter()
        rc = lib.tsne_run(ws)
        if rc != 0:
            raise RuntimeError(f"tsne_run failed ({rc})")
        w3 = time.perf_counter()
        lib.tsne_get_embedding(ws, Yout)
        kl = float(lib.compute_kl_divergence(ws))
        w4 = time.perf_counter()
        run_ms, attr_ms, attr_n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        lib.tsne_get_timing(ws, ctypes.byref(run_ms), ctypes.byref(attr_ms), ctypes.byref(attr_n))
        nr, nl = ctypes.c_int(), ctypes.c_longlong()
        lib.tsne_get_run_stats(ws, ctypes.byref(nr), ctypes.byref(nl))
        lib.tsne_destroy(ws)
        torch.cuda.synchronize()
        w5 = time.perf_counter()
        wall = w5 - w0
        parts = {"host_P": w1 - w0, "init_with_P": w2 - w1, "run": w3 - w2, "get_embedding_kl": w4 - w3,
                 "destroy": w5 - w4}
        return wall, run_ms.value / 1e3, attr_ms.value, attr_n.value, nl.value, nr.value, kl, parts

    def stage_split():
        """The engine's own per-stage device times of one more run (its profiling CSV, the
        reference's schema): attractive pass + update, H2 rebuild, H2 product + force, other."""
        import tempfile
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        with tempfile.TemporaryDirectory() as td:
            f = Path(td) / "stages.csv"
            prm = params_for(be, n, args.iters, args.h2_tol)
            prm.enable_profiling = 1
            prm.profiling_output_file = str(f).encode()
            ws = lib.tsne_init_with_P(None, n, 0, d, ctypes.byref(prm), scipy_csr_to_c_sparse_matrix(P, lib))
            if not ws or lib.tsne_run(ws) != 0:
                raise RuntimeError("profiled run failed")
            lib.tsne_destroy(ws)
            st = O.ref_profile_csv(f)
        return {"attractive": round(float(st["p_matvec"].sum()), 3),
                "h2_rebuild": round(float(st["h2_rebuild"].sum()), 3),
                "h2_product": round(float((st["h2_matvec_s"] + st["h2_matvec_v"] + st["z_computation"]).sum()), 3),
                "other": round(float((st["gradient"] + st["other"]).sum()), 3)}

    for _ in range(args.warmup):
        step()
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    torch.cuda.nvtx.range_push("timed")   # lets a profiler select the timed steps' launches
    res = [step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ck = clocks.stop()
    if dist:
        tdist.barrier()
    dev_s = float(np.mean([r[1] for r in res]))
    wall_s = float(np.mean([r[0] for r in res]))
    if dist:
        from tsne_h2pack._replicas import max_over_ranks
        dev_s, wall_s = max_over_ranks([dev_s, wall_s], device=f"cuda:{local}")
    attr_ms = sum(r[2] for r in res) / max(1, sum(r[3] for r in res))
    launches = int(sum(r[4] for r in res))
    kl = res[-1][6]
    if args.save_embedding and rank == 0:
        np.save(args.save_embedding, Yout)

    out = None
    if rank == 0:
        peaks = json.loads(PEAKS.read_text()) if PEAKS.exists() else {}
        peak = peaks.get("hbm_gbs", 6650.0)
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        attr_bytes = 8.0 * (nnz) + 4.0 * (n + 1) + 28.0 * d * n
        achieved = attr_bytes / (attr_ms * 1e-3) / 1e9
        ratio = traffic_ratio() if d == 2 else None   # the committed capture is of the 2D kernel
        traffic = round(ratio * attr_bytes) if ratio else None
        h2d = 4 * (n + 1) + 12 * nnz + 8 * d * n
        d2h = 8 * d * n + 8
        out = {
            "metric": metric_name(n, args.iters, d), "value": round(dev_s, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dev_s * 1e3, 2), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": data_desc(n, args.seed),
            "config": {"workload": f"{n:,} points x 50 dims -> {d}D, {args.iters} iterations, perplexity 30, "
                                   f"h2_tol {args.h2_tol:g}, H2 rebuild every 3 (10 early), leaf 100, init random",
                       "n_points": n, "nnz_P": int(nnz), "iterations": args.iters,
                       "l2": f"inputs larger than L2 (P streams {8 * nnz / 1e9:.2f} GB per iteration)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": f"{ATTR_FORMS[attr_form(d)]}: attractive CSR pass + gains/momentum update",
                         "avg_launch_ms": round(attr_ms, 4), "algorithmic_bytes": attr_bytes,
                         "peak_source": peak_src},
            "e2e": {"value": round(wall_s, 4), "unit": "s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "breakdown_s": {k: round(float(np.mean([r[7][k] for r in res])), 4) for k in res[0][7]}},
            "gpu_launches": launches,
            "kl_divergence": round(kl, 5),
            "n_rebuild": res[-1][5],
            "setup_s": round(setup_s, 1),
            "split_s": stage_split() if world == 1 else None,
        }
        if ck:
            out["clocks"] = ck
        if not args.no_cpu_baseline and world == 1 and d == 2:
            cb, Y_ref, kl_ref = cpu_sample(P, n, args.iters)
            out["cpu_baseline"] = cb
            if Y_ref is not None:
                out["parity_vs_reference"] = parity(G, P, Yout, kl, Y_ref, kl_ref)
    return out


PUBLISHED_SPLIT = {"attractive": 7.8, "h2_rebuild": 10.7, "h2_product": 8.5, "other": 0.9,
                   "source": "reference benchmarks/results/REPORT.md:205 (Zheng 1M, 2D, 12 threads of an "
                             "Apple M5 Max, H2Pack's own construction; not this hardware or data)"}


def ref_full_run(P, n, iters, warm=False):
    """The reference's own tsne_run over the whole schedule (its sources compiled in
    oracle/_ref: attractive pass, rebuild schedule, fused H2 product, Z identity, update,
    renumbering, KL) on all host cores, on the benchmark's P and init. H2Pack's partition and
    bases, which are absent, are the oracle's restatement behind the H2Pack interface. Times
    tsne_run alone (the reference's "Total optimization time") and reads the reference's own
    per-stage profile. warm: iterations 0-2 only (a warm-up)."""
    import tempfile
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.ref_available():
        raise RuntimeError("oracle/_ref is not built")
    cores = os.cpu_count() or 1
    Y0 = O.init_embedding(n, 2, 1)
    tm = {}
    with tempfile.TemporaryDirectory() as td:
        f = Path(td) / "stages.csv"
        Y, kl = O.ref_run(P, Y0, 3 if warm else iters, learning_rate=max(n / 12.0, 200.0), h2=True,
                          nthreads=cores, attr_f32=2, profile=f, timing=tm)
        st = O.ref_profile_csv(f)
    split = {"attractive": float(st["p_matvec"].sum()), "h2_rebuild": float(st["h2_rebuild"].sum()),
             "h2_product": float((st["h2_matvec_s"] + st["h2_matvec_v"] + st["z_computation"]).sum()),
             "other": float((st["gradient"] + st["other"]).sum())}
    return {"run_s": tm["run_s"], "split_s": {k: round(v, 2) for k, v in split.items()}, "kl": float(kl),
            "Y": Y, "cores": cores}


def ref_sample_text(n, iters):
    return (f"one whole {iters}-iteration run of the reference's own tsne_run (built from its sources in "
            f"oracle/_ref; H2Pack's partition and bases, absent, restated by the oracle) on the {n:,}-point "
            f"workload's P and init, all host cores; timed: tsne_run alone")


def cpu_sample(P, n, iters):
    """CPU baseline on all host cores: a whole run of the reference's own loop (oracle/_ref)
    when it was built, else a bounded sample of the oracle port (an estimate, labelled so).
    Returns (cpu_baseline dict, reference embedding or None, reference KL or None)."""
    try:
        r = ref_full_run(P, n, iters)
    except Exception as e:   # the reference build is absent or failed: time the port
        out = _port_sample(P, n, iters)
        out["sample"] += f" (the reference's own loop was unavailable: {str(e)[:120]})"
        return out, None, None
    out = {"value": round(r["run_s"], 2), "unit": "s", "cores": r["cores"], "kind": "reference",
           "sample": ref_sample_text(n, iters), "split_s": r["split_s"], "kl_divergence": round(r["kl"], 5),
           "published_split_s": PUBLISHED_SPLIT}
    return out, r["Y"], r["kl"]


def quality(G, P, Y, k_list=(10, 30), n_eval=5000, n_anchors=1000):
    """The reference's quality scores (benchmarks/quality.py:56-90): k-NN preservation of
    n_eval seeded query points (the input-space neighbours are the first k of the exact
    graph, the embedding's from a KD-tree) and the common-P KL with Z estimated from
    n_anchors seeded anchor rows. Y: (2, n)."""
    from sklearn.neighbors import KDTree
    n = P.shape[0]
    Yp = np.ascontiguousarray(np.asarray(Y, dtype=np.float64).T)
    rng = np.random.default_rng(0)
    queries = rng.choice(n, size=min(n_eval, n), replace=False)
    k_g = np.diff(G.indptr)
    out = {}
    tree = KDTree(Yp)
    ld = tree.query(Yp[queries], k=max(k_list) + 1, return_distance=False)[:, 1:]
    for k in k_list:
        hits = 0
        for r, i in enumerate(queries):
            a, b = G.indptr[i], G.indptr[i + 1]
            hd = G.indices[a:b][np.argsort(G.data[a:b], kind="stable")[:k]]
            hits += len(set(hd.tolist()) & set(ld[r, :k].tolist()))
        out[f"knn{k}"] = hits / (k * len(queries))
    assert k_g.min() >= max(k_list)
    rows = np.repeat(np.arange(n), np.diff(P.indptr))
    d2 = np.zeros(P.nnz)
    for c in range(Yp.shape[1]):
        d2 += (Yp[rows, c] - Yp[P.indices, c]) ** 2
    anchors = rng.choice(n, size=min(n_anchors, n), replace=False)
    sums = np.empty(len(anchors))
    for a, i in enumerate(anchors):
        w = 1.0 / (1.0 + np.sum((Yp - Yp[i]) ** 2, axis=1))
        w[i] = 0.0
        sums[a] = w.sum()
    Z = n * sums.mean()
    p = P.data
    out["kl_common_P"] = float(np.sum(p * np.log(np.maximum(p, 1e-300))) + np.sum(p * np.log1p(d2)) + np.log(Z))
    return out


def parity(G, P, Y_ours, kl_ours, Y_ref, kl_ref):
    """Final-state parity of the engine's run with the reference loop's run on the same P and
    init: in-run KL within 1%, common-P KL within 1%, 30-NN preservation within 0.5 points."""
    qo, qr = quality(G, P, Y_ours), quality(G, P, Y_ref)
    out = {"kl_run": {"ours": round(kl_ours, 5), "reference": round(kl_ref, 5),
                      "rel_diff": round((kl_ours - kl_ref) / kl_ref, 5)},
           "kl_common_P": {"ours": round(qo["kl_common_P"], 5), "reference": round(qr["kl_common_P"], 5),
                           "rel_diff": round((qo["kl_common_P"] - qr["kl_common_P"]) / qr["kl_common_P"], 5)}}
    for k in (10, 30):
        out[f"knn{k}_preservation"] = {"ours": round(qo[f"knn{k}"], 4), "reference": round(qr[f"knn{k}"], 4),
                                       "diff_points": round(100 * (qo[f"knn{k}"] - qr[f"knn{k}"]), 2)}
    out["pass"] = bool(abs(out["kl_run"]["rel_diff"]) <= 0.01 and abs(out["kl_common_P"]["rel_diff"]) <= 0.01
                       and abs(out["knn30_preservation"]["diff_points"]) <= 0.5)
    out["criteria"] = "KL (in-run and common-P) within 1%, 30-NN preservation within 0.5 points of the reference run"
    return out


def _port_sample(P, n, iters):
    """Bounded CPU sample of the same workload on the oracle port (all host cores):
    iterations 0 and 1 (each an H2 build + product + attractive/update pass) and one more
    attractive pass; the phase estimate uses the schedule's counts (rebuilds, passes)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    Y0 = O.init_embedding(n, 2, 1)
    r = O.Runner(P, Y0, nthreads=cores, n_iter=iters)
    t0 = time.perf_counter(); r.run(0, 1); t1 = time.perf_counter(); r.run(1, 2); t2 = time.perf_counter()
    r.close()
    ta = time.perf_counter(); O.attractive(P, Y0, 12.0, nthreads=cores); tb = time.perf_counter()
    t_pass = tb - ta
    t_rb = max(0.0, 0.5 * ((t1 - t0) + (t2 - t1)) - t_pass)
    n_rb = rebuild_count(iters)
    est = n_rb * t_rb + iters * t_pass
    return {"value": round(est, 2), "unit": "s", "cores": cores, "kind": "port",
            "sample": f"oracle (C/OpenMP FP64 port) iterations 0-1 of the {n:,}-point workload plus one attractive "
                      f"pass ({t2 - t0 + t_pass:.1f} s); estimate = {n_rb} x (H2 build + product "
                      f"{t_rb:.2f} s) + {iters} x pass {t_pass:.3f} s"}


def _job_inputs(specs, device, zipf=False):
    """P of each (n, clusters, perplexity, low_dim, seed, k) job: a 50-dim float32 mixture
    (equal clusters, centres N(0, 5^2), unit noise; or with zipf, the 1M workload's recipe:
    100 Zipf(1.1) clusters, centres N(0, 3^2), per-dimension std U(0.5, 2)), exact k-NN graph on
    the GPU, device calibration (setup, untimed)."""
    from tsne_h2pack._backend import get_backend
    from tsne_h2pack._synthetic import knn_graph_torch, mixture_equal, mixture_zipf
    be = get_backend()
    out = []
    for n, c, perp, d, seed, k in specs:
        if zipf:
            X, _ = mixture_zipf(n, seed=seed)
        else:
            X, _ = mixture_equal(n, n_clusters=c, dim=50, seed=seed, dtype=np.float32)
        G = knn_graph_torch(X, min(k, n - 1), device=f"cuda:{device}")
        out.append((be.joint_P(G, perp), d, perp))
    return out


def _job_params(be, n, iters, perp, seed):
    p = be.create_default_params()
    p.n_iter = iters
    p.verbose = 0
    p.perplexity = perp
    p.learning_rate = max(n / 12.0, 200.0)
    p.h2_tol, p.h2_rebuild_freq, p.h2_rebuild_freq_early, p.h2_leaf_size = 1e-2, 3, 10, 100
    p.random_seed = seed
    p.init_method = 0
    return p


def _serial_plain(be, inputs, iters):
    """The same jobs one after another through the plain C ABI path; per-job latency."""
    from tsne_h2pack._backend import scipy_csr_to_c_sparse_matrix
    lib = be._lib
    lat = []
    for i, (P, d, perp) in enumerate(inputs):
        n = P.shape[0]
        t0 = time.perf_counter()
        prm = _job_params(be, n, iters, perp, i)
        ws = lib.tsne_init_with_P(None, n, 0, d, ctypes.byref(prm), scipy_csr_to_c_sparse_matrix(P, lib))
        if not ws or lib.tsne_run(ws) != 0:
            raise RuntimeError("plain job failed")
        Y = np.zeros((d, n))
        lib.tsne_get_embedding(ws, Y)
        lib.tsne_destroy(ws)
        lat.append(time.perf_counter() - t0)
    return lat


def _pretuned(args, inputs):
    """With --autotune: a leaf-size tuner whose buckets (those of the jobs) are measured during
    setup, outside the timed region."""
    if not args.autotune:
        return None
    from tsne_h2pack.autotune import LeafTuner
    tuner = LeafTuner()
    for P, d, perp in inputs:
        tuner.leaf_for(P.shape[0], d, 1e-2 if d == 2 else 3e-2)
    return tuner


def _pcts(x):
    x = np.asarray(x)
    return {"p50": round(float(np.percentile(x, 50)), 4), "p95": round(float(np.percentile(x, 95)), 4),
            "p99": round(float(np.percentile(x, 99)), 4)}


def batched(args, local):
    """Batched form: J embeddings, N log-uniform in [2000, 50000], 5-30 equal clusters,
    perplexity from {10, 30, 50}, k = 3 perplexity, 2D, 750 iterations, all submitted at once
    to the job server; against the same jobs run one after another (plain path)."""
    import torch
    from tsne_h2pack._backend import get_backend
    from tsne_h2pack.serving import EmbeddingServer
    torch.cuda.set_device(local)
    be = get_backend()
    rng = np.random.default_rng(1234)
    specs = []
    for j in range(args.jobs):
        n = int(round(np.exp(rng.uniform(np.log(2000), np.log(50000)))))
        perp = float(rng.choice([10.0, 30.0, 50.0]))
        specs.append((n, int(rng.integers(5, 31)), perp, 2, 1000 + j, int(3 * perp)))
    iters = 750
    t0 = time.time()
    inputs = _job_inputs(specs, local)
    tuner = _pretuned(args, inputs)
    setup = time.time() - t0
    for i in range(min(3, len(inputs))):   # warm-up (allocator pool, module load)
        _serial_plain(be, inputs[i:i + 1], 50)
    clocks = Clocks(local)
    clocks.start()
    with EmbeddingServer(args.max_concurrent, args.hbm_budget_gb, autotune=tuner or False) as srv:
        t0 = time.perf_counter()
        ids = [srv.submit(P, n_components=d, params=_job_params(be, P.shape[0], iters, perp, i))
               for i, (P, d, perp) in enumerate(inputs)]
        res = [srv.wait(j)[1] for j in ids]
        wall = time.perf_counter() - t0
    ck = clocks.stop()
    assert all(r.ok for r in res)
    t1 = time.perf_counter()
    lat_serial = _serial_plain(be, inputs, iters)
    wall_serial = time.perf_counter() - t1
    value = len(inputs) / wall
    out = {"metric": f"batched jobs/s ({len(inputs)} embeddings, N 2K-50K, {iters} iters, 2D)",
           "value": round(value, 3), "unit": "jobs/s", "n_gpus": 1, "steps": 1, "warmup": 3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic: equal-cluster 50-dim float32 mixtures, seed 1234; exact k = 3 perplexity graphs",
           "config": {"workload": "batched", "jobs": len(inputs), "max_concurrent": args.max_concurrent,
                      "autotune": {f"{d}D 2^{b}": leaf for (d, b), leaf in tuner.table.items()} if tuner else False,
                      "hbm_budget_gb": args.hbm_budget_gb, "iterations": iters,
                      "n_points_total": int(sum(P.shape[0] for P, _, _ in inputs))},
           "serial_plain": {"value": round(len(inputs) / wall_serial, 3), "unit": "jobs/s",
                            "latency_s": _pcts(lat_serial)},
           "speedup_vs_serial": round(wall_serial / wall, 3),
           "latency_s": _pcts([r.latency_s for r in res]), "wall_s": round(wall, 3),
           "setup_s": round(setup, 1)}
    if ck:
        out["clocks"] = ck
    return out


def fit(args, local):
    """End to end from the features: TSNE(knn_method='cuda', init='random').fit_transform(X) on
    the benchmark mixture (n x 50 float32), i.e. the exact k = 90 graph on the device, P
    calibrated, symmetrised and normalised on the device, the optimisation phase, the
    embedding back on the host. Host wall time per fit; the reference publishes 69.3 s for the
    same stages at 1M points (k-NN 34.8 + setup 6.8 + optimisation 27.8 s, Zheng 1M, 12 threads of
    an Apple M5 Max, benchmarks/results/REPORT.md:143)."""
    import torch
    from tsne_h2pack import TSNE
    from tsne_h2pack._synthetic import mixture_zipf
    torch.cuda.set_device(local)
    n = args.n
    X, _ = mixture_zipf(n, seed=1)
    times, kl = [], None
    for i in range(args.warmup + args.steps):
        t = TSNE(n_components=2, perplexity=30.0, max_iter=args.iters, init="random", random_state=1,
                 knn_method="cuda", verbose=0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t.fit_transform(X)
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
        kl = float(t.kl_divergence_)
    v = float(np.mean(times))
    return {"metric": f"fit_transform s at {n:,} pts 2D (k-NN + P + optimisation)", "value": round(v, 3),
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v * 1e3, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": data_desc(n).replace("exact k=90 graph", "exact k=90 graph built inside the timed fit"),
            "config": {"workload": "fit", "n_points": n, "iterations": args.iters, "knn_method": "cuda",
                       "init": "random"},
            "kl_divergence": round(kl, 5),
            "reference_published_s": {"value": 69.3, "parts": {"knn": 34.8, "setup": 6.8, "optimisation": 27.8},
                                      "source": "reference benchmarks/results/REPORT.md:143 (Zheng 1M, 12 threads "
                                                "of an Apple M5 Max; not this hardware or data)"}}


def served(args, local):
    """Served form: Poisson arrivals at `rate` jobs/s for `duration` s; N log-uniform in
    [5000, 200000], 2D (80%) or 3D (20%), 50-dim float32 Zipf mixtures, k = 90, perplexity 30,
    1000 iterations; jobs submitted at their arrival times to the job server. Reports jobs/s
    and p50/p95/p99 latency (arrival to result), and the same jobs run serially."""
    import torch
    from tsne_h2pack._backend import get_backend
    from tsne_h2pack.serving import EmbeddingServer
    torch.cuda.set_device(local)
    be = get_backend()
    rng = np.random.default_rng(4321)
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / args.rate)
        if t > args.duration:
            break
        arrivals.append(t)
    specs = []
    for j in range(len(arrivals)):
        n = int(round(np.exp(rng.uniform(np.log(5000), np.log(200000)))))
        d = 2 if rng.uniform() < 0.8 else 3
        specs.append((n, int(rng.integers(5, 31)), 30.0, d, 5000 + j, 90))
    iters = 1000
    t0 = time.time()
    inputs = _job_inputs(specs, local, zipf=True)
    tuner = _pretuned(args, inputs)
    setup = time.time() - t0
    for i in range(min(2, len(inputs))):
        _serial_plain(be, inputs[i:i + 1], 50)
    clocks = Clocks(local)
    clocks.start()
    with EmbeddingServer(args.max_concurrent, args.hbm_budget_gb, autotune=tuner or False) as srv:
        start = time.perf_counter()
        ids = []
        for i, ((P, d, perp), at) in enumerate(zip(inputs, arrivals)):
            delay = start + at - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(P, n_components=d, params=_job_params(be, P.shape[0], iters, perp, i)))
        res = [srv.wait(j)[1] for j in ids]
        wall = time.perf_counter() - start
    ck = clocks.stop()
    assert all(r.ok for r in res)
    lat_serial = _serial_plain(be, inputs, iters)
    out = {"metric": f"served jobs/s (Poisson {args.rate}/s for {args.duration:.0f} s, N 5K-200K, {iters} iters)",
           "value": round(len(inputs) / wall, 3), "unit": "jobs/s", "n_gpus": 1, "steps": 1, "warmup": 2,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic: 50-dim float32 Zipf(1.1) mixtures, seed 4321; exact k = 90 graphs",
           "config": {"workload": "served", "jobs": len(inputs), "rate": args.rate, "duration_s": args.duration,
                      "autotune": {f"{d}D 2^{b}": leaf for (d, b), leaf in tuner.table.items()} if tuner else False,
                      "max_concurrent": args.max_concurrent, "hbm_budget_gb": args.hbm_budget_gb,
                      "iterations": iters},
           "latency_s": _pcts([r.latency_s for r in res]), "queue_s": _pcts([r.queue_s for r in res]),
           "serial_plain": {"value": round(len(inputs) / sum(lat_serial), 3), "unit": "jobs/s",
                            "run_s": _pcts(lat_serial)},
           "wall_s": round(wall, 3), "setup_s": round(setup, 1)}
    if ck:
        out["clocks"] = ck
    return out


def rebuild_count(iters, freq=3, early=10, exag_iter=250):
    c = 1
    for it in range(1, iters):
        eff = 1 if it < 20 else freq
        if 20 <= it < exag_iter:
            eff = max(eff, early)
        c += it % eff == 0
    return c


def reference(args, rank, world, local):
    """The reference arm: whole runs of the reference's own loop on the host cores. A step is
    a whole 1000-iteration run (about a minute on 16 cores at 1M points), so the arm times
    --ref-runs of them (default 1) after a warm-up of iterations 0-2, whatever --steps and
    --warmup ask, and says so in the line."""
    if rank != 0:
        return None
    if args.dim != 2:
        return {"impl": "reference", "metric": metric_name(args.n, args.iters, args.dim),
                "unavailable": "the reference arm times the 2D workload (the headline metric)"}
    n = args.n
    X, G, P = workload(n, device=local, cache=args.graph_cache)
    ref_full_run(P, n, args.iters, warm=True)
    runs = [ref_full_run(P, n, args.iters) for _ in range(max(1, args.ref_runs))]
    v = float(np.mean([r["run_s"] for r in runs]))
    cb = {"value": round(v, 2), "unit": "s", "cores": runs[0]["cores"], "kind": "reference",
          "sample": ref_sample_text(n, args.iters), "split_s": runs[-1]["split_s"],
          "kl_divergence": round(runs[-1]["kl"], 5), "published_split_s": PUBLISHED_SPLIT}
    return {"impl": "reference", "metric": metric_name(n, args.iters), "value": round(v, 2), "unit": "s",
            "n_gpus": world, "steps": len(runs), "warmup": 1, "steps_requested": args.steps,
            "warmup_requested": args.warmup,
            "steps_note": "a step is one whole optimisation phase of the reference loop on the host cores; the arm "
                          "times --ref-runs of them (default 1) after one warm-up of iterations 0-2, so that the "
                          "command ends within a few minutes",
            "ms_per_step": round(v * 1e3, 1), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": data_desc(n),
            "config": {"workload": f"{n:,} points x 50 dims -> 2D, {args.iters} iterations, perplexity 30, "
                                   "h2_tol 1e-2, H2 rebuild every 3 (10 early), leaf 100, init random",
                       "n_points": n, "iterations": args.iters, "parallelism": "host cores"},
            "cpu_baseline": cb, "e2e": {"value": round(v, 2), "unit": "s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.workload != "plain":
            fn = {"batched": batched, "served": served, "fit": fit}[args.workload]
            out = fn(args, local) if rank == 0 else None
        else:
            out = ours(args, rank, world, local) if args.impl == "ours" else reference(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
