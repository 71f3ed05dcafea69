"""Real-data harness: Leiden on a scanpy connectivity export, scored against
scanpy's own partitions and an annotation (examples/real_data.rs).

An export directory (tools/export_h5ad.py:90-125 in the reference) holds
`indptr.bin` (u64 little-endian), `indices.bin` (u32), `data.bin` (f32) — the
connectivities CSR scanpy clustered — plus `meta.json` and `reference.json`
(scanpy's labels, cluster count and seconds per resolution, optionally an
annotation). The same graph goes to `leiden` at every resolution scanpy ran,
so any difference is the algorithm, not graph construction.

    python -m sc_gpu.real_data <export-dir>
"""
from __future__ import annotations

import json
import math
import os
import sys
import time
from collections import Counter

import numpy as np


def load_export(path: str):
    """(meta, reference, indptr u64, indices u32, data f32) of an export directory."""
    with open(os.path.join(path, "meta.json")) as f:
        meta = json.load(f)
    with open(os.path.join(path, "reference.json")) as f:
        reference = json.load(f)
    indptr = np.fromfile(os.path.join(path, "indptr.bin"), dtype="<u8")
    indices = np.fromfile(os.path.join(path, "indices.bin"), dtype="<u4")
    data = np.fromfile(os.path.join(path, "data.bin"), dtype="<f4")
    return meta, reference, indptr, indices, data


def _pairs(x: float) -> float:
    return x * (x - 1.0) / 2.0


def adjusted_rand_index(a, b) -> float:
    """Adjusted Rand index of two labellings (1 = identical partitions, ~0 =
    chance), from the contingency table's pair counts (real_data.rs:49-76)."""
    a = [int(x) for x in a]
    b = [int(x) for x in b]
    n = float(len(a))
    if n == 0.0:
        return 1.0
    joint = Counter(zip(a, b))
    sum_ij = sum(_pairs(float(c)) for c in joint.values())
    sum_a = sum(_pairs(float(c)) for c in Counter(a).values())
    sum_b = sum(_pairs(float(c)) for c in Counter(b).values())
    total = _pairs(n)
    expected = sum_a * sum_b / total if total else 0.0
    top = 0.5 * (sum_a + sum_b)
    if abs(top - expected) < 1e-12:
        return 1.0
    return (sum_ij - expected) / (top - expected)


def nmi(a, b) -> float:
    """Normalised mutual information, arithmetic-mean normalisation
    (2 I(a; b) / (H(a) + H(b)), real_data.rs:78-110)."""
    a = [int(x) for x in a]
    b = [int(x) for x in b]
    n = float(len(a))
    if n == 0.0:
        return 1.0
    ca, cb = Counter(a), Counter(b)
    mi = 0.0
    for (i, j), c in Counter(zip(a, b)).items():
        p = c / n
        mi += p * math.log(p / ((ca[i] / n) * (cb[j] / n)))

    def entropy(counts):
        return -sum((c / n) * math.log(c / n) for c in counts.values() if c > 0)

    ha, hb = entropy(ca), entropy(cb)
    return 1.0 if ha + hb == 0.0 else 2.0 * mi / (ha + hb)


def run(path: str, out=print) -> list:
    """The harness of examples/real_data.rs on the GPU; returns one dict per
    resolution (ours and scanpy's cluster count, ARI / NMI against scanpy,
    both modularities, both times)."""
    import sc_gpu

    meta, reference, indptr, indices, data = load_export(path)
    out(f"dataset {meta.get('dataset')} — {meta.get('n_cells')} cells, {meta.get('n_entries')} directed "
        f"entries, {meta.get('n_neighbors')}-NN, scanpy {meta.get('scanpy')}")
    t = time.perf_counter()
    graph = sc_gpu.CSRNetwork.from_csr_parts(indptr, indices, data)
    build = time.perf_counter() - t
    out(f"graph built in {build * 1e3:.1f} ms: {graph.node_count()} nodes, {graph.edge_count()} undirected edges, "
        f"self-loops: {graph.has_self_loops()}")
    graph.validate_symmetry()
    out("exhaustive symmetry check: OK")

    annotation = None
    if "annotation" in reference:
        ann = reference["annotation"]
        annotation = [max(int(v), 0) for v in ann["labels"]]
        out(f"author annotation '{ann.get('name')}': {len(ann.get('categories', []))} cell types")

    out("")
    out(f"{'res':>6} | {'ours_k':>7} {'scanpy_k':>8} | {'ARI':>7} {'NMI':>7} | {'ourQ':>8} {'scanpyQ':>8} | "
        f"{'ours(ms)':>9} {'scanpy(ms)':>10}")
    out("-" * 96)
    # the keys are kept as written (Python wrote "1.0", a float would print "1")
    keys = sorted(reference["resolutions"].keys(), key=float)
    rows = []
    best = (0.0, None)
    scanpy_best = 0.0
    for key in keys:
        res = float(key)
        entry = reference["resolutions"][key]
        theirs = [int(v) for v in entry["labels"]]
        t = time.perf_counter()
        c = sc_gpu.leiden(graph, sc_gpu.LeidenConfig.with_resolution(res))
        ms = (time.perf_counter() - t) * 1e3
        ours = c.labels()
        row = {"resolution": res, "ours_k": c.n_clusters(), "scanpy_k": int(entry["n_clusters"]),
               "ari": adjusted_rand_index(ours, theirs), "nmi": nmi(ours, theirs),
               "ours_q": sc_gpu.modularity(graph, ours, res),
               "scanpy_q": sc_gpu.modularity(graph, np.asarray(theirs, np.uint64), res),
               "ours_ms": ms, "scanpy_ms": float(entry["seconds"]) * 1e3}
        rows.append(row)
        out(f"{key:>6} | {row['ours_k']:>7} {row['scanpy_k']:>8} | {row['ari']:>7.4f} {row['nmi']:>7.4f} | "
            f"{row['ours_q']:>8.4f} {row['scanpy_q']:>8.4f} | {ms:>9.1f} {row['scanpy_ms']:>10.1f}")
        if annotation is not None:
            ari = adjusted_rand_index(ours, annotation)
            row["ari_annotation"] = ari
            if ari > best[0]:
                best = (ari, res)
            scanpy_best = max(scanpy_best, adjusted_rand_index(theirs, annotation))
    if annotation is not None:
        out("")
        out(f"best agreement with author cell types: ours ARI {best[0]:.4f} (at resolution {best[1]}), "
            f"scanpy ARI {scanpy_best:.4f}")
    return rows


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print("usage: python -m sc_gpu.real_data <export-dir>", file=sys.stderr)
        return 2
    run(argv[0])
    return 0


if __name__ == "__main__":
    sys.exit(main())
