"""Benchmark: Leiden RB(1.0), seed 7, on the 4M-node Gaussian kNN graph.

Workload (the large single-graph configuration): 4,000,000 points x 30 dims
f32 from a 100-component Gaussian mixture (sigma ~ U[0.7, 1.5], centres
N(0, 4I)); exact kNN k = 10; Gaussian connectivities with per-point sigma =
distance to the k-th neighbour; union-symmetrised u32 / f32 CSR handed over
with from_csr_parts. A "step" is one full leiden() call on that graph.

  value      undirected edges / s of leiden() with the graph resident in HBM
             (edge_count / device time of the run, CUDA events on the
             library's stream), summed over ranks (replicas only: a single
             graph does not shard).
  e2e        the same metric through the public C ABI with host buffers:
             from_csr_parts (H2D + device finish) + leiden + labels D2H.
  cpu_baseline  the CPU oracle (single-threaded restatement of the
             reference's Leiden) on the same graph.

  sweep      (also in the line) the resolution x seed sweep on the 1M x 50
             Gaussian kNN graph (60 components, k = 15): 32 RB resolutions
             log-spaced in [0.1, 3] x 4 seeds = 128 instances, timed as 128
             sequential plain runs and as warm-started chains on concurrent
             streams; speed-up and per-instance modularity differences.
  many_graphs (also in the line, skipped with the sweep) 512 independent
             planted-partition graphs (n log-uniform in [100, 50,000]) in one
             batch call: sequential vs concurrent workers, identical labels.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--n POINTS] [--no-sweep] [--no-cpu-baseline]
  python bench.py --part knn [--n POINTS] [--steps K] [--warmup W] [--knn-precision bf16|fp8]
             times the kNN graph builder alone (points/s) on the same data.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "single-clustering_b200"))

import numpy as np  # noqa: E402

N_POINTS = 4_000_000
DIMS = 30
COMPONENTS = 100
K = 10
GRAPH_SEED = 7
LEIDEN_SEED = 7
METRIC = "Leiden s/run & edges/s @4M nodes (dQ<=1e-3); sweep+warm-start vs plain GPU"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------- workload
def knn_graph_torch(n, d, comps, seed, k, device):
    """Synthetic input only: exact fp32 brute-force kNN with torch, Gaussian
    weights with sigma = k-th neighbour distance, union symmetrisation."""
    import torch
    from sc_gpu import synth
    X, _ = synth.gaussian_mixture(n, d, comps, seed, sigma=(0.7, 1.5))
    x = torch.from_numpy(X).to(device)
    torch.backends.cuda.matmul.allow_tf32 = False
    norms = (x * x).sum(1)
    idx = torch.empty((n, k + 1), dtype=torch.int64, device=device)
    dist = torch.empty((n, k + 1), dtype=torch.float32, device=device)
    chunk = 512
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        d2 = norms[s:e, None] + norms[None, :] - 2.0 * (x[s:e] @ x.T)
        v, i = torch.topk(d2, k + 1, dim=1, largest=False, sorted=True)
        idx[s:e] = i
        dist[s:e] = v.clamp_min_(0).sqrt_()
    sig = dist[:, k]
    rows = torch.arange(n, device=device).repeat_interleave(k)
    cols = idx[:, 1:].reshape(-1)
    dd = dist[:, 1:].reshape(-1)
    si, sj = sig[rows], sig[cols]
    den = si * si + sj * sj
    w = torch.sqrt(2 * si * sj / den) * torch.exp(-dd * dd / den)
    keep = rows != cols
    rows, cols, w = rows[keep], cols[keep], w[keep]
    lo, hi = torch.minimum(rows, cols), torch.maximum(rows, cols)
    key = lo * n + hi
    key, order = torch.sort(key, stable=True)
    w = w[order]
    first = torch.ones_like(key, dtype=torch.bool)
    first[1:] = key[1:] != key[:-1]
    key, w = key[first], w[first]
    lo, hi = key // n, key % n
    r = torch.cat([lo, hi])
    c = torch.cat([hi, lo])
    ww = torch.cat([w, w]).float()
    k2, order = torch.sort(r * n + c)
    r, c, ww = r[order], c[order], ww[order]
    ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(torch.bincount(r, minlength=n), 0)
    out = (ptr.cpu().numpy().astype(np.uint64), c.to(torch.int32).cpu().numpy().view(np.uint32).copy(),
           ww.cpu().numpy())
    del x, norms, idx, dist
    torch.cuda.empty_cache()
    return out


def knn_graph_sc(n, d, comps, seed, k, device_index):
    """The library's own kNN builder: exact search (BF16 tcgen05 candidates +
    FP32 re-rank), sigma = k-th distance, union symmetrisation."""
    import sc_gpu
    from sc_gpu import synth
    X, _ = synth.gaussian_mixture(n, d, comps, seed, sigma=(0.7, 1.5))
    t = time.perf_counter()
    r = sc_gpu.knn_gaussian(X, k, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    KNN_INFO["seconds"] = time.perf_counter() - t
    KNN_INFO["stats"] = sc_gpu.last_run_stats(device_index)
    return r.conn_ptrs, r.conn_nbrs, r.conn_w


KNN_INFO = {}

SWEEP_POINTS, SWEEP_DIMS, SWEEP_COMPONENTS, SWEEP_K, SWEEP_SEED = 1_000_000, 50, 60, 15, 11
SWEEP_RESOLUTIONS = 32
SWEEP_SEEDS = (1, 2, 3, 4)


def run_sweep(device_index, n_points=SWEEP_POINTS, n_streams=16, split=2):
    """128-instance resolution x seed sweep: sequential plain runs vs
    warm-started chains (each seed's chain cut in `split` pieces whose heads
    start from the seed's finest partition) on concurrent streams."""
    import sc_gpu
    from sc_gpu import synth
    X, _ = synth.gaussian_mixture(n_points, SWEEP_DIMS, SWEEP_COMPONENTS, SWEEP_SEED, sigma=(0.7, 1.5))
    r = sc_gpu.knn_gaussian(X, SWEEP_K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    g = sc_gpu.CSRNetwork.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w, device=device_index)
    del X, r
    res = np.geomspace(0.1, 3.0, SWEEP_RESOLUTIONS)
    sc_gpu.leiden(g)  # warm-up of the sequential arm
    # warm-up of the concurrent arm: its workers' temporaries settle in the
    # device pool (16 instances at once need more than one run leaves there)
    sc_gpu.leiden_sweep(g, res, SWEEP_SEEDS, warm_start=True, n_streams=n_streams, split=split)
    out = {}
    for name, warm, streams in (("plain_sequential", False, 1), ("warm_chains", True, n_streams)):
        t = time.perf_counter()
        sw = sc_gpu.leiden_sweep(g, res, SWEEP_SEEDS, warm_start=warm, n_streams=streams, split=split if warm else 1)
        dt = time.perf_counter() - t
        out[name] = (dt, {k: sc_gpu.modularity(g, v.labels(), k[0]) for k, v in sw.items()})
    base_s, base_q = out["plain_sequential"]
    warm_s, warm_q = out["warm_chains"]
    d = np.array([warm_q[k] - base_q[k] for k in base_q])
    return {"workload": f"sweep_rb{SWEEP_RESOLUTIONS}x{len(SWEEP_SEEDS)}_knn{SWEEP_K}_gmm{n_points}x{SWEEP_DIMS}",
            "instances": len(base_q), "edge_count": g.edge_count(), "plain_sequential_s": base_s,
            "warm_chains_s": warm_s, "streams": n_streams, "chain_split": split, "speedup": base_s / warm_s,
            "dQ_min": float(d.min()), "dQ_mean": float(d.mean()), "dQ_max": float(d.max()),
            "frac_dQ_ge_-1e-4": float(np.mean(d >= -1e-4))}


MANY_GRAPHS, MANY_SEED, MANY_STREAMS = 512, 21, 16


def run_many_graphs(device_index, count=MANY_GRAPHS, n_streams=MANY_STREAMS):
    """512 independent planted-partition graphs (node counts log-uniform in
    [100, 50,000], 5-200 blocks, mean degree U[10, 30], 80% of the draws inside
    the block, f32 weights U[0.5, 1.5]), RB(1) seed 42 on each: one batch call
    with sequential instances vs one with concurrent workers. The labels of
    the two must be identical (a fixed seed is bit-reproducible)."""
    import sc_gpu
    from sc_gpu import synth
    graphs = []
    nodes = edges = 0
    for n, src, dst, w, _ in synth.many_planted_graphs(count, MANY_SEED):
        g = sc_gpu.CSRNetwork.from_edge_arrays(n, src, dst, w, device=device_index)
        graphs.append(g)
        nodes += n
        edges += g.edge_count()
    cfgs = [sc_gpu.LeidenConfig(objective=sc_gpu.Rb(1.0), seed=42)] * count
    sc_gpu.leiden_batch(graphs, cfgs, n_streams=n_streams)  # warm-up: workers' temporaries settle in the pool
    t = time.perf_counter()
    seq = sc_gpu.leiden_batch(graphs, cfgs, n_streams=1)
    seq_s = time.perf_counter() - t
    t = time.perf_counter()
    bat = sc_gpu.leiden_batch(graphs, cfgs, n_streams=n_streams)
    bat_s = time.perf_counter() - t
    same = all(a == b for a, b in zip(seq, bat))
    return {"workload": f"many_planted{count}_n100-50000", "graphs": count, "nodes": nodes, "edges": edges,
            "sequential_s": seq_s, "batched_s": bat_s, "streams": n_streams, "speedup": seq_s / bat_s,
            "graphs_per_s": count / bat_s, "edges_per_s": edges / bat_s, "labels_identical": bool(same)}


def run_knn_part(args, device_index):
    """The kNN graph builder alone on the bench's point set."""
    import sc_gpu
    from sc_gpu import synth
    prec = sc_gpu.KNN_FP8 if args.knn_precision == "fp8" else sc_gpu.KNN_BF16
    X, _ = synth.gaussian_mixture(args.n, DIMS, COMPONENTS, GRAPH_SEED, sigma=(0.7, 1.5))
    for _ in range(args.warmup):
        sc_gpu.knn_gaussian(X, K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, precision=prec, device=device_index)
    t = time.perf_counter()
    for _ in range(args.steps):
        r = sc_gpu.knn_gaussian(X, K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, precision=prec,
                                device=device_index)
    dt = (time.perf_counter() - t) / args.steps
    line = {"metric": f"kNN graph build points/s (exact k=10, {args.knn_precision.upper()} tcgen05 candidates "
                      "+ FP32 re-rank)",
            "value": args.n / dt, "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "dtype": args.knn_precision, "data": "synthetic",
            "config": {"workload": f"knn{K}_gmm{args.n}x{DIMS}", "n_points": args.n, "dims": DIMS, "k": K},
            "timing": "host wall clock around the C ABI call (host input, host CSR output)",
            "conn_nnz": int(len(r.conn_w))}
    if not args.no_cpu_baseline:
        line["cpu_baseline"], line["recall_at_k"] = knn_cpu_baseline(X, r.index)
    print(json.dumps(line), flush=True)


def knn_cpu_baseline(X, gpu_index, sample=20000):
    """Substitute CPU baseline (the reference's kd-tree / HNSW crates cannot be
    built here): scikit-learn's exact kd-tree search on all host cores, timed on
    a bounded query sample and scaled to points/s; its neighbours also give the
    GPU result's recall@k on that sample."""
    from sklearn.neighbors import NearestNeighbors
    n = X.shape[0]
    rng = np.random.Generator(np.random.PCG64(0))
    q = np.sort(rng.choice(n, min(sample, n), replace=False))
    t = time.perf_counter()
    nn = NearestNeighbors(n_neighbors=K + 1, algorithm="kd_tree", n_jobs=-1).fit(X)
    build = time.perf_counter() - t
    t = time.perf_counter()
    _, idx = nn.kneighbors(X[q])
    dt = time.perf_counter() - t
    per_point = dt / len(q)
    hits = sum(len(set(a.tolist()) & set(b.tolist())) for a, b in zip(gpu_index[q], idx))
    return ({"value": 1.0 / (per_point + build / n), "unit": "points/s", "cores": os.cpu_count(),
             "kind": "substitute: scikit-learn kd-tree, exact", "sample": f"{len(q)} queries against all {n} points, "
             "tree build amortised over n", "build_s": build, "query_s": dt}, hits / idx.size)


def make_graph(args, device):
    if args.graph == "lattice":
        from sc_gpu import synth
        return synth.knn_like_graph(args.n, k=K, seed=GRAPH_SEED)
    if args.graph == "gmm-torch":
        return knn_graph_torch(args.n, DIMS, COMPONENTS, GRAPH_SEED, K, device)
    return knn_graph_sc(args.n, DIMS, COMPONENTS, GRAPH_SEED, K, device.index or 0)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        mx = max(float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()) if sm else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 5 + i and s[5 + i].lower() in ("active", "0x1", "1")})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


# ---------------------------------------------------------------- arms
def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_cpu_baseline(ptr, nbr, w, seed):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    g = O.Graph.from_csr_parts(ptr, nbr, w)
    t = time.perf_counter()
    lab, ncl = g.leiden(seed=seed, resolution=1.0)
    dt = time.perf_counter() - t
    return g, lab, dt


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_POINTS)
    ap.add_argument("--graph", default="gmm", choices=["gmm", "gmm-torch", "lattice"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--sweep-points", type=int, default=SWEEP_POINTS)
    ap.add_argument("--part", default="leiden", choices=["leiden", "knn"])
    ap.add_argument("--knn-precision", default="bf16", choices=["bf16", "fp8"])
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = torch.device("cuda", local_rank)

    workload = {"workload": f"leiden_rb1_seed{LEIDEN_SEED}_knn{K}_gmm{args.n}x{DIMS}",
                "n_points": args.n, "dims": DIMS, "components": COMPONENTS, "k": K,
                "graph": args.graph, "sigma": "kth", "symmetrisation": "union",
                "objective": "rb", "resolution": 1.0, "seed": LEIDEN_SEED,
                "l2": "inputs larger than L2 (graph > 126 MB)", "parallelism": f"replicas{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            if dist:
                dist.destroy_process_group()
            return
        ptr, nbr, w = make_graph(args, device)
        g, lab, dt = run_cpu_baseline(ptr, nbr, w, LEIDEN_SEED)
        m = g.edge_count()
        eps = m / dt
        line = {"metric": METRIC, "value": eps, "unit": "edges/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "ms_per_step": dt * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload,
                "modularity": g.modularity(lab),
                "cpu_baseline": {"value": eps, "unit": "edges/s", "cores": 1, "kind": "port",
                                 "sample": "one full leiden() run on the whole graph",
                                 "cpu": cpu_model(), "nproc": os.cpu_count()},
                "e2e": {"value": eps, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    if args.part == "knn":
        if rank == 0:
            run_knn_part(args, local_rank)
        if dist:
            dist.destroy_process_group()
        return

    import sc_gpu
    t0 = time.perf_counter()
    ptr, nbr, w = make_graph(args, device)
    log(f"graph built in {time.perf_counter() - t0:.1f}s: n={len(ptr) - 1} entries={len(nbr)}")
    g = sc_gpu.CSRNetwork.from_csr_parts(ptr, nbr, w, device=local_rank)
    m = g.edge_count()
    cfg = sc_gpu.LeidenConfig(objective=sc_gpu.Rb(1.0), seed=LEIDEN_SEED)

    for _ in range(args.warmup):
        sc_gpu.leiden(g, cfg)
    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_ms = 0.0
    stats = None
    t = time.perf_counter()
    for _ in range(args.steps):
        c = sc_gpu.leiden(g, cfg)
        stats = sc_gpu.last_run_stats(local_rank)
        dev_ms += stats["ms_total"]
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms_step = dev_ms / args.steps
    if dist:
        tt = torch.tensor([ms_step], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_step = float(tt.item())
    value = world * m / (ms_step / 1e3)
    q = sc_gpu.modularity(g, c.labels())

    # e2e through the C ABI with host buffers
    torch.cuda.synchronize()
    t = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 2))
    graph_s = leiden_s = 0.0
    e2e_each = []
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        g2 = sc_gpu.CSRNetwork.from_csr_parts(ptr, nbr, w, device=local_rank)
        t2 = time.perf_counter()
        c2 = sc_gpu.leiden(g2, cfg)
        t3 = time.perf_counter()
        graph_s += t2 - t1
        leiden_s += t3 - t2
        dev_ms = sc_gpu.last_run_stats(local_rank)["ms_total"]
        del g2
        e2e_each.append({"graph_upload_s": t2 - t1, "leiden_call_s": t3 - t2, "graph_free_s": time.perf_counter() - t3,
                         "leiden_device_ms": dev_ms})
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t) / e2e_steps
    h2d = ptr.nbytes + nbr.nbytes + w.nbytes
    d2h = len(ptr) * 8 - 8

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    hbm, peak_kind = peaks()
    lm_gbs = stats["alg_bytes_local_move"] / (stats["ms_local_move"] / 1e3) / 1e9 if stats["ms_local_move"] else 0
    line = {"metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload,
            "s_per_run": ms_step / 1e3, "edge_count": m, "modularity": q, "n_clusters": c.n_clusters(),
            "wall_s_per_step": wall / args.steps,
            "phases_ms": {k: stats[k] for k in ("ms_local_move", "ms_refine", "ms_aggregate", "ms_other")},
            "run_stats": {k: stats[k] for k in ("passes", "levels", "local_move_sweeps", "moves")},
            "gpu_launches": int(stats["kernel_launches"]) * args.steps,
            "roofline": {"bound": "hbm", "kernel": "local-move sweeps (decide + apply)",
                         "achieved": lm_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": lm_gbs / hbm if hbm else None, "traffic": None,
                         "peak_kind": peak_kind},
            "clocks": clk,
            "e2e": {"value": world * m / e2e_s, "unit": "edges/s", "s_per_run": e2e_s,
                    "graph_upload_s": graph_s / e2e_steps, "leiden_call_s": leiden_s / e2e_steps,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "each": e2e_each}}
    if KNN_INFO:
        line["knn_graph_build_s"] = KNN_INFO["seconds"]
    if not args.no_sweep:
        del g
        line["sweep"] = run_sweep(local_rank, args.sweep_points)
        line["many_graphs"] = run_many_graphs(local_rank)
    if not args.no_cpu_baseline:
        og, lab_o, dt = run_cpu_baseline(ptr, nbr, w, LEIDEN_SEED)
        q_o = og.modularity(lab_o)
        line["cpu_baseline"] = {"value": m / dt, "unit": "edges/s", "cores": 1, "kind": "port",
                                "sample": "one full leiden() run of the CPU oracle on the same graph",
                                "s_per_run": dt, "modularity": q_o, "cpu": cpu_model(),
                                "nproc": os.cpu_count()}
        line["dQ_vs_cpu"] = q - q_o
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
