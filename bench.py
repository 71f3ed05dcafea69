"""Benchmark: Leiden RB(1.0), seed 7, on the 4M-node Gaussian kNN graph.

Workload (the large single-graph configuration): 4,000,000 points x 30 dims
f32 from a 100-component Gaussian mixture (sigma ~ U[0.7, 1.5], centres
N(0, 4I)); exact kNN k = 10; Gaussian connectivities with per-point sigma =
distance to the k-th neighbour; union-symmetrised u32 / f32 CSR handed over
with from_csr_parts. A "step" is one full leiden() call on that graph. The
graph is built with torch alone (synth.knn_graph_exact_torch, an exact FP64
search), identically in both arms, so the reference arm never loads this
library; the library's own kNN builder is timed on the same points beside it
(`library_knn`: build time, recall@k and connectivity error against FP64).

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

  c2         (also in the line) 200,000 x 50 points, 30 components, k = 15:
             the graph from FP32 CUDA-core and from BF16 tensor-core candidate
             distances (both re-ranked in FP32), recall and connectivity error
             of each, Leiden RB 1.0 and CPM 0.05 on each, the CPU oracle's
             quality on the same graphs.
  c5         (also in the line) 2,000,000 x 50 points, 200 components, k = 15
             from FP8 e4m3 candidates (BF16 beside it): recall, then the edge
             MLP trained at RB {0.5, 1, 2} and evaluated as a warm start at
             RB {0.8, 1.5} against the plain start.
  cpu_baseline.calibration  the CPU oracle on the reference benchmark's own
             100k-node shape beside its published ~110 ms.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--n POINTS] [--no-sweep] [--no-c2] [--no-c5] [--no-accuracy]
                  [--no-cpu-baseline]
  python bench.py --part knn [--n POINTS] [--steps K] [--warmup W] [--knn-precision bf16|fp8]
             times the kNN graph builder alone (points/s) on the same data.
  python bench.py --part c5          the 2M x 50 FP8 kNN + learned warm start leg alone
  python bench.py --part mlp --n N   a few training epochs and one proposal on N points (ncu)
  python bench.py --part once --n N  one leiden() run on the library's kNN graph of N points (ncu)

  Under torchrun (N > 1) every rank also runs the sweep's warm chains dealt
  across the ranks (`sweep.sharded`, max over ranks).
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
    KNN_INFO["points"] = X
    KNN_INFO["index"] = r.index
    return r.conn_ptrs, r.conn_nbrs, r.conn_w


KNN_INFO = {}

SWEEP_POINTS, SWEEP_DIMS, SWEEP_COMPONENTS, SWEEP_K, SWEEP_SEED = 1_000_000, 50, 60, 15, 11
SWEEP_RESOLUTIONS = 32
SWEEP_SEEDS = (1, 2, 3, 4)


def run_sweep(device_index, n_points=SWEEP_POINTS, n_streams=16, split=8, accuracy=True, warm_passes=1):
    """128-instance resolution x seed sweep: sequential plain runs vs
    warm-started chains (each seed's chain cut in `split` pieces whose heads
    start from the seed's finest partition; a warm-started instance runs
    `warm_passes` passes) on concurrent streams."""
    import sc_gpu
    from sc_gpu import synth
    X, _ = synth.gaussian_mixture(n_points, SWEEP_DIMS, SWEEP_COMPONENTS, SWEEP_SEED, sigma=(0.7, 1.5))
    r = sc_gpu.knn_gaussian(X, SWEEP_K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    acc = (knn_accuracy(X, r.index, r.conn_ptrs, r.conn_nbrs, r.conn_w, SWEEP_K, f"cuda:{device_index}")
           if accuracy else None)
    g = sc_gpu.CSRNetwork.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w, device=device_index)
    del X, r
    res = np.geomspace(0.1, 3.0, SWEEP_RESOLUTIONS)
    sc_gpu.leiden(g)  # warm-up of the sequential arm
    # warm-up of the concurrent arm: its workers' temporaries settle in the
    # device pool (16 instances at once need more than one run leaves there)
    sc_gpu.leiden_sweep(g, res, SWEEP_SEEDS, warm_start=True, n_streams=n_streams, split=split,
                        warm_passes=warm_passes)
    out = {}
    times = {}
    for name, warm, streams in (("plain_sequential", False, 1), ("warm_chains", True, n_streams)):
        times[name] = []
        for _ in range(2):  # host-side scheduling varies from call to call: the best of two, both reported
            t = time.perf_counter()
            sw = sc_gpu.leiden_sweep(g, res, SWEEP_SEEDS, warm_start=warm, n_streams=streams,
                                     split=split if warm else 1, warm_passes=warm_passes)
            times[name].append(time.perf_counter() - t)
        out[name] = (min(times[name]), {k: sc_gpu.modularity(g, v.labels(), k[0]) for k, v in sw.items()})
    # the same warm-started chains as batched device work: each wave of instances
    # whose warm start is done runs over the disjoint union of their graphs
    sc_gpu.leiden_sweep(g, res, SWEEP_SEEDS, warm_start=True, split=split, warm_passes=warm_passes, union=True)
    times["warm_union"] = []
    for _ in range(2):
        t = time.perf_counter()
        sw = sc_gpu.leiden_sweep(g, res, SWEEP_SEEDS, warm_start=True, split=split, warm_passes=warm_passes,
                                 union=True)
        times["warm_union"].append(time.perf_counter() - t)
    out["warm_union"] = (min(times["warm_union"]), {k: sc_gpu.modularity(g, v.labels(), k[0]) for k, v in sw.items()})
    base_s, base_q = out["plain_sequential"]
    warm_s, warm_q = out["warm_chains"]
    uni_s, uni_q = out["warm_union"]
    du = np.array([uni_q[k] - base_q[k] for k in base_q])
    d = np.array([warm_q[k] - base_q[k] for k in base_q])
    return {"workload": f"sweep_rb{SWEEP_RESOLUTIONS}x{len(SWEEP_SEEDS)}_knn{SWEEP_K}_gmm{n_points}x{SWEEP_DIMS}",
            "instances": len(base_q), "edge_count": g.edge_count(), "plain_sequential_s": base_s,
            "warm_chains_s": warm_s, "streams": n_streams, "chain_split": split, "warm_passes": warm_passes,
            "plain_passes": 2, "speedup": base_s / warm_s, "times_s": times,
            "dQ_min": float(d.min()), "dQ_mean": float(d.mean()), "dQ_max": float(d.max()),
            "frac_dQ_ge_-1e-4": float(np.mean(d >= -1e-4)),
            "union": {"s": uni_s, "speedup": base_s / uni_s, "dQ_min": float(du.min()), "dQ_max": float(du.max()),
                      "frac_dQ_ge_-1e-4": float(np.mean(du >= -1e-4)),
                      "how": "waves of warm-started instances, each wave one disjoint-union run"},
            "knn_accuracy": acc}


def run_sweep_sharded(device_index, rank, world, dist, n_points=SWEEP_POINTS, n_streams=16, warm_passes=1):
    """The sweep's warm-started chains dealt across the ranks by cost (one
    chain per seed: parallel.run_sharded), each rank running its share on its
    own GPU; the only collective is one all-gather of the instances'
    modularities after the runs. The kNN graph is built split by query rows
    (parallel.knn_sharded), timed on its own. Both timed from a barrier, max
    over ranks."""
    import torch
    import sc_gpu
    from sc_gpu import parallel, synth
    X, _ = synth.gaussian_mixture(n_points, SWEEP_DIMS, SWEEP_COMPONENTS, SWEEP_SEED, sigma=(0.7, 1.5))
    # the kNN graph split by query rows (parallel.knn_sharded): each rank
    # searches its block against all points, one all-gather of the lists, then
    # every rank builds the connectivities (the single build's bits)
    sc_gpu.knn_search(X[:4096], SWEEP_K, 0, 4096, device=device_index)  # warm-up
    dist.barrier()
    torch.cuda.synchronize()
    t = time.perf_counter()
    idx, d2 = parallel.knn_sharded(lambda b, e: sc_gpu.knn_search(X, SWEEP_K, b, e, device=device_index),
                                   n_points, rank, world)
    r = sc_gpu.knn_connectivities(idx, d2, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    torch.cuda.synchronize()
    tk = torch.tensor([time.perf_counter() - t], dtype=torch.float64, device=f"cuda:{device_index}")
    dist.all_reduce(tk, op=dist.ReduceOp.MAX)
    g = sc_gpu.CSRNetwork.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w, device=device_index)
    del X, r, idx, d2
    res = np.geomspace(0.1, 3.0, SWEEP_RESOLUTIONS)
    configs, warm, keys = sc_gpu.sweep_plan(res, SWEEP_SEEDS, sc_gpu.Rb, True, None, 8, warm_passes)
    cost = [3.0 if w < 0 else 1.0 for w in warm]  # a singleton start costs about three warm runs
    timing = {}

    def run_local(ids, local_warm):
        timing["instances"] = len(ids)
        if not ids:  # more ranks than chains: this rank idles
            timing["s"] = 0.0
            return []
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = sc_gpu.leiden_batch([g] * len(ids), [configs[i] for i in ids], local_warm, n_streams)
        timing["s"] = time.perf_counter() - t
        timing["instances"] = len(ids)
        return [sc_gpu.modularity(g, c.labels(), keys[i][0]) for i, c in zip(ids, out)]

    sc_gpu.leiden_batch([g] * 4, configs[:4], warm[:4], n_streams)  # warm-up
    dist.barrier()
    qs = parallel.run_sharded(run_local, len(configs), warm, cost, rank, world)
    tt = torch.tensor([timing["s"]], dtype=torch.float64, device=f"cuda:{device_index}")
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return {"workload": f"sweep_rb{SWEEP_RESOLUTIONS}x{len(SWEEP_SEEDS)}_knn{SWEEP_K}_gmm{n_points}x{SWEEP_DIMS}",
            "ranks": world, "s": float(tt.item()), "instances": len(configs),
            "knn_sharded_s": float(tk.item()),
            "knn_how": "parallel.knn_sharded: row blocks searched per rank (full scan), one all-gather of the "
                       "k+1 lists, connectivities on every rank",
            "instances_rank0": timing["instances"], "units": "one warm chain per seed (its 8 pieces concurrent on the rank's streams), dealt by cost",
            "q_min": float(min(qs)), "q_max": float(max(qs)),
            "how": "parallel.run_sharded: no collective inside a run, one all-gather of modularities"}


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
    sc_gpu.leiden_batch(graphs, cfgs, union=True)  # warm-up
    uni_s = []
    for _ in range(2):
        t = time.perf_counter()
        uni = sc_gpu.leiden_batch(graphs, cfgs, union=True)
        uni_s.append(time.perf_counter() - t)
    st = sc_gpu.last_run_stats(device_index)
    same_u = all(a == b for a, b in zip(seq, uni))
    return {"workload": f"many_planted{count}_n100-50000", "graphs": count, "nodes": nodes, "edges": edges,
            "sequential_s": seq_s, "batched_s": bat_s, "streams": n_streams, "speedup": seq_s / bat_s,
            "graphs_per_s": count / bat_s, "edges_per_s": edges / bat_s, "labels_identical": bool(same),
            "union": {"s": min(uni_s), "times_s": uni_s, "speedup": seq_s / min(uni_s),
                      "graphs_per_s": count / min(uni_s), "edges_per_s": edges / min(uni_s),
                      "labels_identical_to_sequential": bool(same_u), "device_ms": st["ms_total"],
                      "kernel_launches": int(st["kernel_launches"]),
                      "how": "all 512 graphs as one disjoint union: every launch covers every instance"}}


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
            "conn_nnz": int(len(r.conn_w)), "pruning": sc_gpu.knn_last_stats(device_index)}
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


# ---------------------------------------------------------------- kNN accuracy
def fp64_knn(Xd, nrm, rows, k, device, block=64, margin=8):
    """Exact FP64 k+1 nearest points (self included) of the points `rows` of the
    device array Xd (float64): candidates from the norm-expanded FP64 distances
    with a margin, then exact FP64 differences ordered by (distance, self first,
    index). Returns host (idx int64, dist float64), len(rows) x (k+1)."""
    import torch
    n = Xd.shape[0]
    kk = min(n, k + 1 + margin)
    out_i = np.empty((len(rows), k + 1), np.int64)
    out_d = np.empty((len(rows), k + 1), np.float64)
    for s in range(0, len(rows), block):
        r = torch.from_numpy(np.asarray(rows[s:s + block], np.int64)).to(device)
        d2 = nrm[r, None] + nrm[None, :] - 2.0 * (Xd[r] @ Xd.T)
        _, cand = torch.topk(d2, kk, dim=1, largest=False)
        del d2
        dd = ((Xd[cand] - Xd[r][:, None, :]) ** 2).sum(-1)
        cand, dd, rr = cand.cpu().numpy(), dd.cpu().numpy(), r.cpu().numpy()
        order = np.lexsort((cand, cand != rr[:, None], dd), axis=-1)[:, : k + 1]
        out_i[s:s + block] = np.take_along_axis(cand, order, 1)
        out_d[s:s + block] = np.sqrt(np.take_along_axis(dd, order, 1))
    return out_i, out_d


def knn_accuracy(X, index, ptrs, nbrs, w, k, device, sample=2000, seed=0):
    """recall@k of the library's k-nearest lists and the largest connectivity
    error against an FP64 exact search, on `sample` seeded query points.

    recall_at_k         |library's k neighbours (self excluded) & FP64's| / k
    recall_at_k_ties    the same, a library neighbour whose FP64 distance ties
                        the true k-th within 1e-6 relative counted as a hit
    max_rel_conn_err    over the FP64 neighbours j of each sampled i: the
                        library's CSR weight (i, j) against the FP64 Gaussian
                        weight with sigma = FP64 k-th distance (union
                        symmetrisation, the bench's setting); edges the library
                        lacks are counted in missing_edges instead."""
    import torch
    n = X.shape[0]
    rng = np.random.Generator(np.random.PCG64(seed))
    q = np.sort(rng.choice(n, min(sample, n), replace=False))
    Xd = torch.from_numpy(np.ascontiguousarray(X)).to(device, torch.float64)
    nrm = (Xd * Xd).sum(1)
    t = time.perf_counter()
    ti, td = fp64_knn(Xd, nrm, q, k, device)
    nb = np.unique(ti[:, 1:].reshape(-1))
    si, sd = fp64_knn(Xd, nrm, nb, k, device)
    sig = dict(zip(nb.tolist(), sd[:, k].tolist()))
    hits = hits_t = 0
    max_rel = max_abs = 0.0
    missing = 0
    X64 = X.astype(np.float64)
    for r, i in enumerate(q):
        truth = set(ti[r, 1:].tolist())
        got = [j for j in index[i, 1:].tolist() if j != i]
        kth = td[r, k]
        for j in got:
            if j in truth:
                hits += 1
                hits_t += 1
            else:
                dj = float(np.sqrt(((X64[i] - X64[j]) ** 2).sum()))
                hits_t += abs(dj - kth) <= 1e-6 * max(kth, 1e-30)
        row = nbrs[int(ptrs[i]):int(ptrs[i + 1])]
        for t2 in range(1, k + 1):
            j = int(ti[r, t2])
            s_i, s_j, dist = td[r, k], sig[j], td[r, t2]
            den = s_i * s_i + s_j * s_j
            w64 = np.sqrt(2 * s_i * s_j / den) * np.exp(-dist * dist / den)
            pos = np.searchsorted(row, j)
            if pos >= len(row) or row[pos] != j:
                missing += 1
                continue
            err = abs(float(w[int(ptrs[i]) + pos]) - w64)
            max_abs = max(max_abs, err)
            max_rel = max(max_rel, err / w64)
    del Xd, nrm
    torch.cuda.empty_cache()
    return {"recall_at_k": hits / (len(q) * k), "recall_at_k_ties": hits_t / (len(q) * k),
            "max_rel_conn_err": max_rel, "max_abs_conn_err": max_abs, "missing_edges": missing,
            "sample": f"{len(q)} seeded query points (PCG64 seed {seed}) against all {n}, FP64 exact search "
                      "(torch float64 on the device) incl. the k-th distances of their neighbours",
            "check_s": time.perf_counter() - t}


# ---------------------------------------------------------------- C2
C2_POINTS, C2_DIMS, C2_COMPONENTS, C2_K, C2_SEED = 200_000, 50, 30, 15, 2


def run_c2(device_index, cpu=True):
    """kNN + Gaussian connectivities + Leiden on 200,000 x 50 points of a
    30-component mixture (centres N(0, 4I), sigma 1, Dirichlet(1) weights):
    exact k = 15 with sigma = k-th distance, union symmetrisation; candidates
    from FP32 CUDA-core distances and from BF16 tensor-core distances, both
    re-ranked in exact FP32; Leiden RB 1.0 and CPM 0.05 on each graph, and the
    CPU oracle on the same graphs."""
    import sc_gpu
    from sc_gpu import synth
    X, _ = synth.gaussian_mixture(C2_POINTS, C2_DIMS, C2_COMPONENTS, C2_SEED, sigma=(1.0, 1.0))
    out = {"workload": f"knn{C2_K}_gmm{C2_POINTS}x{C2_DIMS}_c{C2_COMPONENTS}", "sigma": "kth",
           "symmetrisation": "union", "arms": {}}
    csr = {}
    for name, prec in (("fp32", sc_gpu.KNN_FP32), ("bf16", sc_gpu.KNN_BF16)):
        sc_gpu.knn_gaussian(X, C2_K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, precision=prec,
                            device=device_index)  # warm-up
        t = time.perf_counter()
        r = sc_gpu.knn_gaussian(X, C2_K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, precision=prec,
                                device=device_index)
        arm = {"knn_build_s": time.perf_counter() - t, "pruning": sc_gpu.knn_last_stats(device_index),
               "accuracy": knn_accuracy(X, r.index, r.conn_ptrs, r.conn_nbrs, r.conn_w, C2_K,
                                        f"cuda:{device_index}")}
        csr[name] = (r.conn_ptrs, r.conn_nbrs, r.conn_w)
        g = sc_gpu.CSRNetwork.from_csr_parts(*csr[name], device=device_index)
        arm["edge_count"] = g.edge_count()
        for oname, obj in (("rb1.0", sc_gpu.Rb(1.0)), ("cpm0.05", sc_gpu.Cpm(0.05))):
            cfg = sc_gpu.LeidenConfig(objective=obj, seed=42)
            sc_gpu.leiden(g, cfg)
            c = sc_gpu.leiden(g, cfg)
            st = sc_gpu.last_run_stats(device_index)
            res = {"ms": st["ms_total"], "n_clusters": c.n_clusters(),
                   "quality": sc_gpu.quality(g, c.labels(), obj)}
            if oname.startswith("rb"):
                res["modularity"] = sc_gpu.modularity(g, c.labels(), 1.0)
            arm[oname] = res
        out["arms"][name] = arm
    # the kNN autotuner on these points: the full scan against several cluster
    # counts of the pruned search (lists identical), the fastest kept
    out["knn_autotune"] = sc_gpu.knn_autotune(X, C2_K, device=device_index)
    sc_gpu.set_knn_clusters(0, device_index)
    a, b = csr["fp32"], csr["bf16"]
    out["graphs_identical"] = bool(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                                   and np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32)))
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        cb = {}
        for name in ("fp32", "bf16"):
            og = O.Graph.from_csr_parts(*csr[name])
            for oname, kind, gamma in (("rb1.0", O.RB, 1.0), ("cpm0.05", O.CPM, 0.05)):
                t = time.perf_counter()
                lab, ncl = og.leiden(objective=kind, resolution=gamma, seed=42)
                dt = time.perf_counter() - t
                qo = og.quality(lab, kind, gamma)
                gpu = out["arms"][name][oname]
                # quality per unit of total edge weight (modularity's scale for RB)
                tw = og.total_weight()
                cb[f"{name}/{oname}"] = {"s": dt, "quality": qo, "n_clusters": int(ncl),
                                         "dQ_per_weight": (gpu["quality"] - qo) / tw}
        out["cpu_baseline"] = {"kind": "port", "cores": 1, "runs": cb,
                               "sample": "one full leiden() run of the CPU oracle per graph and objective"}
    return out


# ---------------------------------------------------------------- C5
C5_POINTS, C5_DIMS, C5_COMPONENTS, C5_K, C5_SEED = 2_000_000, 50, 200, 15, 5


def run_c5(device_index):
    """Learned warm start + FP8 kNN on 2,000,000 x 50 points of a 200-component
    mixture (sigma U[0.5, 2.0]): kNN k = 15 from FP8 e4m3 per-row-scaled
    candidates re-ranked in FP32 (BF16 candidates beside it for their recall);
    the edge MLP trained on plain-GPU partitions at RB {0.5, 1.0, 2.0}
    (independent seeds), evaluated as a warm start at RB {0.8, 1.5} against the
    plain singleton start, which is also the fallback. The graph carries the
    points as its embedding (the edge-length feature)."""
    import sc_gpu
    from sc_gpu import synth
    from sc_gpu.learned import EdgeMlp, warm_start_leiden
    X, _ = synth.gaussian_mixture(C5_POINTS, C5_DIMS, C5_COMPONENTS, C5_SEED, sigma=(0.5, 2.0))
    dev = f"cuda:{device_index}"
    out = {"workload": f"knn{C5_K}_gmm{C5_POINTS}x{C5_DIMS}_c{C5_COMPONENTS}", "knn": {}}
    keep = None
    for name, prec in (("fp8", sc_gpu.KNN_FP8), ("bf16", sc_gpu.KNN_BF16)):
        t = time.perf_counter()
        r = sc_gpu.knn_gaussian(X, C5_K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, precision=prec,
                                device=device_index)
        out["knn"][name] = {"build_s": time.perf_counter() - t, "pruning": sc_gpu.knn_last_stats(device_index),
                            "accuracy": knn_accuracy(X, r.index, r.conn_ptrs, r.conn_nbrs, r.conn_w, C5_K, dev)}
        if name == "fp8":
            keep = (r.conn_ptrs, r.conn_nbrs, r.conn_w)
        del r
    g = sc_gpu.CSRNetwork.from_csr_parts(*keep, device=device_index)
    del keep
    t = time.perf_counter()
    g.set_embedding(X)  # the points: the model reads edge lengths in their projection
    out["embedding_attach_s"] = time.perf_counter() - t
    del X
    out["edge_count"] = g.edge_count()

    def run(gamma, seed):
        return sc_gpu.leiden(g, sc_gpu.LeidenConfig(objective=sc_gpu.Rb(gamma), seed=seed)).labels()

    sc_gpu.leiden(g)  # warm-up
    t = time.perf_counter()
    labs = {0.5: run(0.5, 101), 1.0: run(1.0, 102), 2.0: run(2.0, 103)}
    alt = {0.5: run(0.5, 201), 2.0: run(2.0, 203)}
    ctx = {0.5: (alt[0.5], labs[1.0]), 1.0: (labs[0.5], labs[2.0]), 2.0: (labs[1.0], alt[2.0])}
    t_part = time.perf_counter() - t
    m = EdgeMlp(seed=4)
    t = time.perf_counter()
    rounds, epochs = 6, 20
    for _ in range(rounds):
        for gamma in (0.5, 1.0, 2.0):
            loss = m.train(g, labs[gamma], gamma, epochs=epochs, lr=5e-3, context=ctx[gamma])
    out["training"] = {"resolutions": [0.5, 1.0, 2.0], "seeds": [101, 102, 103], "calls": 3 * rounds,
                       "epochs_per_call": epochs, "train_s": time.perf_counter() - t, "final_loss": loss,
                       "partition_runs_s": t_part}
    ev = {}
    for gamma, c in ((0.8, (labs[0.5], labs[1.0])), (1.5, (labs[1.0], labs[2.0]))):
        cfg = sc_gpu.LeidenConfig(objective=sc_gpu.Rb(gamma), seed=9)
        warm_start_leiden(m, g, cfg, threshold=0.9, core_fraction=0.0, context=c)  # warm-up
        res = warm_start_leiden(m, g, cfg, threshold=0.9, core_fraction=0.0, context=c)
        ev[str(gamma)] = {"used_proposal": res.used_proposal, "q_warm": res.q_warm, "q_plain": res.q_plain,
                          "dQ": res.q_warm - res.q_plain, "sweeps_warm": res.sweeps_warm,
                          "sweeps_plain": res.sweeps_plain, "ms_warm": res.ms_warm, "ms_plain": res.ms_plain,
                          "ms_saved": res.ms_plain - res.ms_warm, "ms_proposal": res.ms_proposal,
                          "proposal_clusters": res.proposal_clusters}
    out["warm_start"] = ev
    return out


def run_mlp_small(device_index, n_points):
    """The edge MLP on the kNN graph of n_points of the C5 mixture (k = 15, the
    points as the embedding): plain runs for the labels (RB 1) and the context
    (RB 0.5 and 2), 2 training calls of 5 epochs, one proposal; wall times of
    each."""
    import sc_gpu
    from sc_gpu import synth
    from sc_gpu.learned import EdgeMlp
    X, _ = synth.gaussian_mixture(n_points, C5_DIMS, C5_COMPONENTS, C5_SEED, sigma=(0.5, 2.0))
    r = sc_gpu.knn_gaussian(X, C5_K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    g = sc_gpu.CSRNetwork.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w, device=device_index)
    g.set_embedding(X)
    del X, r
    lab = sc_gpu.leiden(g, sc_gpu.LeidenConfig(seed=1)).labels()
    ctx = (sc_gpu.leiden(g, sc_gpu.LeidenConfig(objective=sc_gpu.Rb(0.5), seed=2)).labels(),
           sc_gpu.leiden(g, sc_gpu.LeidenConfig(objective=sc_gpu.Rb(2.0), seed=3)).labels())
    m = EdgeMlp(seed=4, device=device_index)
    out = {"points": n_points, "edges": g.edge_count()}
    t = time.perf_counter()
    for _ in range(2):
        loss = m.train(g, lab, 1.0, epochs=5, lr=5e-3, context=ctx)
    out["train_s"] = time.perf_counter() - t
    out["loss"] = loss
    t = time.perf_counter()
    _, k = m.propose(g, 1.0, 0.9, 0.0, context=ctx)
    out["propose_s"] = time.perf_counter() - t
    out["proposal_clusters"] = k
    return out


def make_graph(args, device):
    """The Leiden input of both arms. "gmm" (default): the exact kNN graph of the
    4M-point mixture built with torch alone (synth.knn_graph_exact_torch), so
    the reference arm never loads this library and both arms cluster the same
    bytes; the library's own kNN builder is timed and checked on the same
    points in a leg of its own. "gmm-sc": the library's kNN graph instead."""
    from sc_gpu import synth
    if args.graph == "lattice":
        return synth.knn_like_graph(args.n, k=K, seed=GRAPH_SEED)
    if args.graph == "gmm-sc":
        return knn_graph_sc(args.n, DIMS, COMPONENTS, GRAPH_SEED, K, device.index or 0)
    X, comp = synth.gaussian_mixture(args.n, DIMS, COMPONENTS, GRAPH_SEED, sigma=(0.7, 1.5))
    t = time.perf_counter()
    ptr, nbr, w, idx, dist = synth.knn_graph_exact_torch(X, comp, K, device)
    GRAPH_INFO["build_s"] = time.perf_counter() - t
    GRAPH_INFO["points"] = X
    return ptr, nbr, w


GRAPH_INFO = {}


def library_knn_leg(X, ptr, nbr, w, device_index, accuracy=True):
    """The library's kNN builder (BF16 tcgen05 candidates + FP32 re-rank,
    sigma = k-th distance, union) on the headline's points: build time, recall
    and connectivity error against FP64, and how its graph compares with the
    exact graph the Leiden runs use."""
    import sc_gpu
    sc_gpu.knn_gaussian(X[:65536], K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    t = time.perf_counter()
    r = sc_gpu.knn_gaussian(X, K, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION, device=device_index)
    out = {"build_s": time.perf_counter() - t, "precision": "bf16", "points": int(X.shape[0]),
           "pruning": sc_gpu.knn_last_stats(device_index)}
    same_ptr = np.array_equal(r.conn_ptrs, ptr)
    same_nbr = same_ptr and np.array_equal(r.conn_nbrs, nbr)
    out["same_edges_as_exact_graph"] = bool(same_nbr)
    if same_nbr:
        rel = np.abs(r.conn_w.astype(np.float64) - w) / np.maximum(w, 1e-30)
        out["max_rel_weight_diff_vs_exact_graph"] = float(rel.max())
    else:
        out["entries"], out["exact_graph_entries"] = int(len(r.conn_nbrs)), int(len(nbr))
    # tensor-core work: one (256-query group, 128-point tile) pair is a
    # 256 x 128 x KA contraction; KA = 32 columns for up to 30 dimensions, else 64
    st = out["pruning"]
    n, d = X.shape
    ka = 32 if d <= 30 else 64
    executed = 2.0 * 256 * 128 * ka * st["tiles_scanned"]
    scan_ms = st["ms_pass1"] + st["ms_pass2"]
    peak, kind = bf16_peak()
    out["flops"] = {"executed": executed, "scan_ms": scan_ms,
                    "executed_tflops": executed / (scan_ms / 1e3) / 1e12 if scan_ms else None,
                    "frac_of_bf16_peak": executed / (scan_ms / 1e3) / 1e12 / peak if scan_ms else None,
                    "full_scan_flops": 2.0 * n * n * d,
                    "full_scan_equivalent_tflops": 2.0 * n * n * d / out["build_s"] / 1e12,
                    "peak_tflops": peak, "peak_kind": kind,
                    "note": "executed: the pruned search's tensor-core FLOPs over its two scan passes; the kernel "
                            "is bound by its candidate epilogue (tensor pipe ~5% active in "
                            "profiles/k_knn_tc_gmm262144x30.md), so the fraction stays small by design"}
    if accuracy:
        out["accuracy"] = knn_accuracy(X, r.index, r.conn_ptrs, r.conn_nbrs, r.conn_w, K, f"cuda:{device_index}")
    return out


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self._proc = None
        self._t = None

    def start(self):
        # one long-lived nvidia-smi sampling every 200 ms: starting a new one
        # per sample initialises NVML each time, and those start-ups stall the
        # driver (and the timed launches) for tens of milliseconds
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._proc = None
            return
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def mark(self):
        """Drops the samples taken so far: only those of the timed region count."""
        self.samples = []

    def _run(self):
        for line in self._proc.stdout:
            out = line.strip()
            if out:
                self.samples.append([x.strip() for x in out.split(",")])

    def stop(self):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except subprocess.TimeoutExpired:
                self._proc.kill()
                self._proc.wait()
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
# DRAM bytes per algorithmic byte of the local-moving phase, from the warm-cache
# ncu capture of a whole run on the 1M-point graph of the same family
# (profiles/local_move_dram_knn10_gmm1000000x30.md: 7.39 GB read + written for
# 3.866 GB algorithmic); the 4M-point run's traffic is this ratio times its
# algorithmic bytes.
LM_TRAFFIC_PER_ALG_BYTE = 7.39 / 3.866


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bf16_peak():
    """Dense BF16 TFLOP/s: the measured burst figure, else the earlier fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def run_cpu_baseline(ptr, nbr, w, seed):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    g = O.Graph.from_csr_parts(ptr, nbr, w)
    t = time.perf_counter()
    lab, ncl = g.leiden(seed=seed, resolution=1.0)
    dt = time.perf_counter() - t
    return g, lab, dt


def blob_knn_graph(n=100_000, blocks=10, k=15, seed=5):
    """The shape of the reference's own Leiden benchmark (benches/leiden.rs:17-68):
    n points in `blocks` squares of side 16 around centres on a circle of radius
    60, each joined to its k nearest points, unit weights, the undirected union
    of those pairs (from_edges). Points are drawn with numpy's PCG64, not the
    reference's ChaCha8, and the neighbours by an exact kd-tree: at this density
    the reference's +-2-cell grid holds every true neighbour."""
    from scipy.spatial import cKDTree
    rng = np.random.Generator(np.random.PCG64(seed))
    per = n // blocks
    b = np.minimum(np.arange(n) // per, blocks - 1)
    a = 2 * np.pi * np.arange(blocks) / blocks
    pts = np.stack([60 * np.cos(a)[b] + rng.random(n) * 16 - 8, 60 * np.sin(a)[b] + rng.random(n) * 16 - 8], 1)
    _, idx = cKDTree(pts).query(pts, k + 1)
    src = np.repeat(np.arange(n), k)
    dst = idx[:, 1:].reshape(-1)
    key = np.unique(np.minimum(src, dst).astype(np.int64) * n + np.maximum(src, dst))
    return n, (key // n).astype(np.uint64), (key % n).astype(np.uint64)


README_MS_100K = 110.0  # README.md:18: "100k nodes / 840k edges in ~110 ms single-threaded"


def cpu_calibration():
    """The CPU oracle on the reference benchmark's 100k-node shape, best of 3,
    beside the reference's published time for it (hardware unstated)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n, src, dst = blob_knn_graph()
    g = O.Graph.from_edges(n, src=src, dst=dst, w=np.ones(len(src)))
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        g.leiden(seed=42)
        ts.append(time.perf_counter() - t)
    best = min(ts) * 1e3
    return {"workload": "benches/leiden.rs knn_graph(100000, 10, 15) shape: 2-D blobs, unit weights",
            "nodes": n, "edges": g.edge_count(), "oracle_ms_best_of_3": best,
            "reference_published_ms": README_MS_100K, "oracle_over_published": best / README_MS_100K,
            "note": "published figure: README.md:18, single-threaded, hardware not stated"}


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
    ap.add_argument("--graph", default="gmm", choices=["gmm", "gmm-sc", "lattice"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-c2", action="store_true", help="skip the 200k x 50 FP32-vs-BF16 configuration")
    ap.add_argument("--no-c5", action="store_true", help="skip the 2M x 50 FP8 + learned warm start configuration")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP64 recall / connectivity checks")
    ap.add_argument("--sweep-points", type=int, default=SWEEP_POINTS)
    ap.add_argument("--part", default="leiden", choices=["leiden", "knn", "once", "c5", "mlp"],
                    help="once: one leiden() run on the library's kNN graph of --n points (a small case for ncu); "
                         "c5: the 2M x 50 FP8 kNN + learned warm start configuration alone; "
                         "mlp: a few training epochs and one proposal on --n points of the C5 mixture (for ncu)")
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
                                 "cpu": cpu_model(), "nproc": os.cpu_count(),
                                 "calibration": cpu_calibration()},
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
    if args.part == "mlp":
        if rank == 0:
            print(json.dumps({"part": "mlp", **run_mlp_small(local_rank, args.n)}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.part == "c5":
        if rank == 0:
            print(json.dumps({"part": "c5", **run_c5(local_rank)}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    if args.part == "once":
        if rank == 0:
            import sc_gpu
            ptr, nbr, w = knn_graph_sc(args.n, DIMS, COMPONENTS, GRAPH_SEED, K, local_rank)
            g = sc_gpu.CSRNetwork.from_csr_parts(ptr, nbr, w, device=local_rank)
            sc_gpu.leiden(g, sc_gpu.LeidenConfig(objective=sc_gpu.Rb(1.0), seed=LEIDEN_SEED))
            print(json.dumps({"part": "once", "n": args.n, "edges": g.edge_count(), "entries": g.entry_count(),
                              **sc_gpu.last_run_stats(local_rank)}), flush=True)
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

    # the routing autotuner on this graph (first level under each candidate
    # routing; labels never depend on it): the timed runs use what it keeps
    tuned = sc_gpu.autotune(g, cfg)

    # the clock sampler starts before the warm-up: its first nvidia-smi calls
    # (driver and NVML start-up) stall the host for a moment, and inside the
    # timed region that stall would leave the GPU idle between launches
    clocks = ClockSampler(local_rank)
    clocks.start()
    for _ in range(args.warmup):
        sc_gpu.leiden(g, cfg)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.mark()
    dev_ms = 0.0
    ms_each = []
    stats = None
    t = time.perf_counter()
    for _ in range(args.steps):
        c = sc_gpu.leiden(g, cfg)
        stats = sc_gpu.last_run_stats(local_rank)
        dev_ms += stats["ms_total"]
        ms_each.append(stats["ms_total"])
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

    # e2e through the C ABI with host buffers. One untimed step first, as for
    # the device-resident loop: the first graph uploaded beside the resident
    # one grows the library's graph pool (a one-time cost per process, measured
    # 0.02-0.3 s on different boxes), which every later upload reuses.
    g2 = sc_gpu.CSRNetwork.from_csr_parts(ptr, nbr, w, device=local_rank)
    sc_gpu.leiden(g2, cfg)
    del g2
    torch.cuda.synchronize()
    t = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
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

    sharded = None
    if dist and not args.no_sweep:
        sharded = run_sweep_sharded(local_rank, rank, world, dist, args.sweep_points)
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
            "wall_s_per_step": wall / args.steps, "ms_each": ms_each,
            "phases_ms": {k: stats[k] for k in ("ms_local_move", "ms_refine", "ms_aggregate", "ms_other")},
            "run_stats": {k: stats[k] for k in ("passes", "levels", "local_move_sweeps", "moves")},
            "autotune": tuned,
            "gpu_launches": int(stats["kernel_launches"]) * args.steps,
            "roofline": {"bound": "hbm", "kernel": "local-move sweeps (decide + apply)",
                         "achieved": lm_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": lm_gbs / hbm if hbm else None,
                         "traffic": LM_TRAFFIC_PER_ALG_BYTE * stats["alg_bytes_local_move"],
                         "algorithmic_bytes": stats["alg_bytes_local_move"],
                         "traffic_note": "DRAM bytes of the phase per run: the warm-cache ncu ratio of the "
                                         "1M-point run (profiles/local_move_dram_knn10_gmm1000000x30.md) x "
                                         "this run's algorithmic bytes",
                         "peak_kind": peak_kind},
            "roofline_phases": {
                ph: {"achieved": stats[f"alg_bytes_{key}"] / (stats[f"ms_{ms}"] / 1e3) / 1e9 if stats[f"ms_{ms}"] else None,
                     "frac": (stats[f"alg_bytes_{key}"] / (stats[f"ms_{ms}"] / 1e3) / 1e9 / hbm
                              if stats[f"ms_{ms}"] and hbm else None),
                     "algorithmic_bytes": stats[f"alg_bytes_{key}"], "ms": stats[f"ms_{ms}"], "unit": "GB/s",
                     "peak": hbm, "peak_kind": peak_kind}
                for ph, key, ms in (("refine", "refine", "refine"), ("aggregate", "aggregate", "aggregate"))},
            "clocks": clk,
            "e2e": {"value": world * m / e2e_s, "unit": "edges/s", "s_per_run": e2e_s,
                    "graph_upload_s": graph_s / e2e_steps, "leiden_call_s": leiden_s / e2e_steps,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "each": e2e_each}}
    if GRAPH_INFO:
        line["input_graph"] = {"builder": "synth.knn_graph_exact_torch (torch only, FP64 exact kNN)",
                               "build_s": GRAPH_INFO["build_s"]}
        line["library_knn"] = library_knn_leg(GRAPH_INFO.pop("points"), ptr, nbr, w, local_rank,
                                              accuracy=not args.no_accuracy)
        line["knn_graph_build_s"] = line["library_knn"]["build_s"]
    if KNN_INFO:
        line["knn_graph_build_s"] = KNN_INFO["seconds"]
        if not args.no_accuracy:
            line["knn_accuracy"] = knn_accuracy(KNN_INFO["points"], KNN_INFO["index"], ptr, nbr, w, K,
                                                f"cuda:{local_rank}")
        KNN_INFO.pop("points")
        KNN_INFO.pop("index")
    if not args.no_sweep:
        del g
        line["sweep"] = run_sweep(local_rank, args.sweep_points, accuracy=not args.no_accuracy)
        if sharded:
            line["sweep"]["sharded"] = sharded
        line["many_graphs"] = run_many_graphs(local_rank)
    if not args.no_c2:
        line["c2"] = run_c2(local_rank, cpu=not args.no_cpu_baseline)
    if not args.no_c5:
        line["c5"] = run_c5(local_rank)
    if not args.no_cpu_baseline:
        og, lab_o, dt = run_cpu_baseline(ptr, nbr, w, LEIDEN_SEED)
        q_o = og.modularity(lab_o)
        line["cpu_baseline"] = {"value": m / dt, "unit": "edges/s", "cores": 1, "kind": "port",
                                "sample": "one full leiden() run of the CPU oracle on the same graph",
                                "s_per_run": dt, "modularity": q_o, "cpu": cpu_model(),
                                "nproc": os.cpu_count(), "calibration": cpu_calibration()}
        line["dQ_vs_cpu"] = q - q_o
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
