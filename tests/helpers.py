"""Graph fixtures and metrics shared by the tests.

Restates the fixtures of single-clustering's tests/common/mod.rs:10-194 and
src/testdata.rs:41-127 (test_graphs, sbm, nmi, disconnected_community_count).
The reference draws its random graphs from ChaCha8; these use numpy's PCG64,
so the graphs have the same shapes but not the same edges.
"""
from __future__ import annotations

import gzip
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def karate():
    with open(os.path.join(GOLDEN, "karate.json")) as f:
        k = json.load(f)
    return [(a, b, 1.0) for a, b in k["edges"]], np.array(k["optimum"], np.uint64)


def leidenalg_fixture():
    with open(os.path.join(GOLDEN, "leidenalg_reference.json.gz"), "rb") as f:
        return json.loads(gzip.decompress(f.read()))


def sbm(n_per, blocks, p_in, p_out, seed):
    """Stochastic block model edge list and planted labels (testdata.rs:41-61)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = n_per * blocks
    truth = np.arange(n) // n_per
    iu, ju = np.triu_indices(n, 1)
    p = np.where(truth[iu] == truth[ju], p_in, p_out)
    keep = rng.random(iu.shape[0]) < p
    edges = [(int(a), int(b), 1.0) for a, b in zip(iu[keep], ju[keep])]
    return edges, truth.astype(np.uint64)


def cliques(n_blocks, size, bridges=()):
    edges = []
    for b in range(n_blocks):
        for i in range(size):
            for j in range(i + 1, size):
                edges.append((b * size + i, b * size + j, 1.0))
    edges.extend((a, c, 1.0) for a, c in bridges)
    return edges


def reference_graphs():
    """(name, n, edges) of tests/common/mod.rs:57-130."""
    k_edges, _ = karate()
    rng = np.random.Generator(np.random.PCG64(3))
    weighted = [(a, b, 0.25 + 3.5 * rng.random()) for a, b, _ in k_edges]
    sbm_edges, _ = sbm(25, 4, 0.35, 0.03, 1)
    return [
        ("empty", 0, []),
        ("single_node", 1, []),
        ("no_edges", 8, []),
        ("one_edge", 2, [(0, 1, 1.0)]),
        ("self_loops_only", 4, [(0, 0, 1.0), (1, 1, 2.0), (2, 2, 0.5)]),
        ("with_self_loops", 5, [(0, 1, 1.0), (1, 2, 1.0), (0, 0, 3.0), (3, 4, 1.0), (3, 3, 2.0)]),
        ("star", 9, [(0, i, 1.0) for i in range(1, 9)]),
        ("path", 12, [(i, i + 1, 1.0) for i in range(11)]),
        ("karate", 34, k_edges),
        ("karate_weighted", 34, weighted),
        ("sbm", 100, sbm_edges),
        ("disconnected_cliques", 15, cliques(3, 5)),
    ]


def random_graph(seed):
    """A randomly shaped graph (tests/properties.rs:21-61)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(rng.integers(1, 121))
    density = rng.random() ** 2 * 0.6 + 0.01
    weighted = bool(rng.integers(0, 2))
    loops = rng.random() < 0.3
    blocks = min(int(rng.integers(2, 7)), n) if rng.integers(0, 2) else 1
    edges = []
    for a in range(n):
        for b in range(a + 1, n):
            same = blocks > 1 and (a * blocks // n) == (b * blocks // n)
            p = density * 4.0 if same else density
            if rng.random() < min(p, 1.0):
                w = 0.05 + 4.0 * rng.random() if weighted else 1.0
                edges.append((a, b, w))
    if loops:
        for v in range(n):
            if rng.random() < 0.2:
                edges.append((v, v, 0.5 + 2.0 * rng.random()))
    return n, edges


def nmi(a, b):
    """Normalized mutual information (testdata.rs:64-100)."""
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    n = float(len(a))
    if n == 0:
        return 1.0
    ka, kb = int(a.max()) + 1, int(b.max()) + 1
    joint = np.zeros((ka, kb))
    np.add.at(joint, (a, b), 1.0)
    pa, pb = joint.sum(1), joint.sum(0)
    p = joint / n
    nz = p > 0
    mi = float(np.sum(p[nz] * np.log(p[nz] / ((pa[:, None] / n) * (pb[None, :] / n))[nz])))

    def h(x):
        x = x[x > 0] / n
        return -float(np.sum(x * np.log(x)))

    ha, hb = h(pa), h(pb)
    return 1.0 if ha + hb == 0 else 2.0 * mi / (ha + hb)


def disconnected_community_count(ptr, nbr, labels):
    """Communities that are not internally connected (testdata.rs:104-127)."""
    n = len(ptr) - 1
    labels = np.asarray(labels, np.int64)
    n_comms = int(labels.max()) + 1 if n else 0
    seen = np.zeros(n, bool)
    comps = np.zeros(n_comms, np.int64)
    for v in range(n):
        if seen[v]:
            continue
        comps[labels[v]] += 1
        stack = [v]
        seen[v] = True
        while stack:
            u = stack.pop()
            for e in range(int(ptr[u]), int(ptr[u + 1])):
                x = int(nbr[e])
                if not seen[x] and labels[x] == labels[u]:
                    seen[x] = True
                    stack.append(x)
    return int(np.sum(comps > 1))


def edges_to_arrays(edges):
    src = np.array([e[0] for e in edges], np.uint64)
    dst = np.array([e[1] for e in edges], np.uint64)
    w = np.array([e[2] for e in edges], np.float64)
    return src, dst, w
