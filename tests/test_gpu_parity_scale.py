"""Bit-exact parity at scale, outside the exact-summation regime, and the
Louvain / weight-cap modes against the oracle.

A 1M-point Gaussian kNN graph carries f32 weights spanning many binades, so
f64 sums of them round and their order matters: aggregation takes its ordered
sort path (segments split across blocks) and the per-community sums of
modularity / quality their ordered chains. Given the oracle's own partitions,
at level 0 and again on the level-1 graph, the GPU's aggregated CSR (ids and
f32 weight bits), node weights, strengths, total weight, partition aggregates,
RB / CPM quality and modularity must equal the oracle's bit for bit
(csr_network.rs:516-608, partition.rs:75-112, objective.rs:108-244).
"""
import numpy as np
import pytest

import oracle as O
import sc_gpu
from sc_gpu import synth
from helpers import karate

pytestmark = pytest.mark.gpu


def bits(x):
    return np.asarray(x, dtype=np.float64).view(np.uint64)


def assert_same_graph(og, gg, what):
    a = og.arrays()
    ptr, nbr, w = gg.to_csr_parts()
    assert np.array_equal(a["ptr"], ptr), what
    assert np.array_equal(a["nbr"], nbr), what
    assert np.array_equal(a["w"].view(np.uint32), w.view(np.uint32)), what
    assert np.array_equal(bits(a["node_w"]), bits(gg.node_weights())), what
    assert np.array_equal(bits(a["strength"]), bits(gg.strengths())), what
    assert bits(a["total_weight"]) == bits(gg.total_weight()), what
    assert a["edge_count"] == gg.edge_count(), what


def outside_exact_regime(w, total):
    """Every f64 sum of these f32 weights is exact only if the total stays below
    2^(52 + e0), e0 the exponent of the lowest set bit over all of them."""
    b = w[w > 0].astype(np.float32).view(np.uint32).astype(np.int64)
    ex = (b >> 23) & 0xFF
    mant = (b & 0x7FFFFF) | np.where(ex > 0, 1 << 23, 0)
    low = np.log2((mant & -mant).astype(np.float64)).astype(np.int64)
    e0 = int(np.min(np.where(ex > 0, ex - 150, -149) + low))
    return total >= 2.0 ** (52 + e0)


def assert_same_evaluation(og, gg, part, what):
    for gamma in (1.0, 0.5):
        assert bits(og.modularity(part, gamma)) == bits(sc_gpu.modularity(gg, part, gamma)), (what, gamma)
    assert bits(og.quality(part, O.RB, 1.0)) == bits(sc_gpu.quality(gg, part, sc_gpu.Rb(1.0))), what
    assert bits(og.quality(part, O.CPM, 0.05)) == bits(sc_gpu.quality(gg, part, sc_gpu.Cpm(0.05))), what
    a = og.partition_stats(part)
    b = gg.partition_stats(part)
    assert np.array_equal(a["size"], b["size"]), what
    for key in ("weight", "strength", "internal"):
        assert np.array_equal(bits(a[key]), bits(b[key])), (what, key)


@pytest.fixture(scope="module")
def knn_million():
    X, _ = synth.gaussian_mixture(1_000_000, 30, 100, seed=17, sigma=(0.7, 1.5))
    r = sc_gpu.knn_gaussian(X, 10, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION)
    return r.conn_ptrs, r.conn_nbrs, r.conn_w


def check_levels(ptrs, nbrs, w):
    og = O.Graph.from_csr_parts(ptrs, nbrs, w)
    gg = sc_gpu.CSRNetwork.from_csr_parts(ptrs, nbrs, w)
    assert_same_graph(og, gg, "level-0 graph")
    # level 0: the oracle's local-moving partition from singletons
    n = og.node_count()
    part0, _ = og.local_move(np.arange(n, dtype=np.uint64), O.RB, 1.0, seed=3)
    assert len(np.unique(part0)) < n // 2
    assert_same_evaluation(og, gg, part0, "level 0")
    oc, gc = og.aggregate(part0), gg.aggregate(part0)
    assert_same_graph(oc, gc, "level-1 graph")
    # level 1: the oracle's partition of its own coarse graph, then the level-2 graph
    n1 = oc.node_count()
    part1, _ = oc.local_move(np.arange(n1, dtype=np.uint64), O.RB, 1.0, seed=4)
    assert_same_evaluation(oc, gc, part1, "level 1")
    assert_same_graph(oc.aggregate(part1), gc.aggregate(part1), "level-2 graph")
    # a coarse grouping with very long segments (a few huge communities)
    coarse = (part0 % 7).astype(np.uint64)
    assert_same_evaluation(og, gg, coarse, "7 groups")
    assert_same_graph(og.aggregate(coarse), gg.aggregate(coarse), "7-group graph")
    return gg


def test_bit_exact_on_a_million_point_knn_graph(knn_million):
    """The Gaussian kNN graph itself (sigma = k-th distance keeps every weight in
    about [0.3, 1]): inside the exact regime, where aggregation may take its
    hashed contraction path."""
    ptrs, nbrs, w = knn_million
    gg = check_levels(ptrs, nbrs, w)
    assert not outside_exact_regime(w, gg.total_weight())


def test_bit_exact_outside_the_exact_regime_at_scale(knn_million):
    """The same graph with every weight raised to the 40th power (still
    symmetric, now spanning some 70 binades): f64 sums round, so aggregation
    takes the ordered sort path with long segments split across blocks, and the
    per-community sums their ordered chains."""
    ptrs, nbrs, w = knn_million
    w40 = np.power(w.astype(np.float64), 40).astype(np.float32)
    keep = w40 > 0
    assert keep.all()
    gg = check_levels(ptrs, nbrs, w40)
    assert outside_exact_regime(w40, gg.total_weight())


def _planted():
    src, dst, w, _ = synth.planted_partition()
    og = O.Graph.from_edges(20000, src=src, dst=dst, w=w)
    gg = sc_gpu.CSRNetwork.from_edge_arrays(20000, src, dst, w)
    return og, gg


def _knn(n=60000):
    X, _ = synth.gaussian_mixture(n, 50, 200, 5, sigma=(0.5, 2.0))
    r = sc_gpu.knn_gaussian(X, 15, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION)
    og = O.Graph.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w)
    gg = sc_gpu.CSRNetwork.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w)
    return og, gg


@pytest.mark.parametrize("which", ["planted20k", "knn60k"])
@pytest.mark.parametrize("gamma", [0.5, 1.0, 2.0])
def test_louvain_mode_quality_against_the_oracle(which, gamma):
    """refine = false (leiden/mod.rs:245-257): the level collapses by the working
    partition itself. Bar: Q >= oracle Q - 1e-3 at the same resolution."""
    og, gg = _planted() if which == "planted20k" else _knn()
    lab_o, _ = og.leiden(objective=O.RB, resolution=gamma, seed=42, refine=False)
    q_o = og.modularity(lab_o, gamma)
    c = sc_gpu.leiden(gg, sc_gpu.LeidenConfig(objective=sc_gpu.Rb(gamma), seed=42, refine=False))
    q = sc_gpu.modularity(gg, c.labels(), gamma)
    assert q >= q_o - 1e-3, (q, q_o)
    # labels consecutive from 0, as Clustering::from_normalized
    assert set(np.unique(c.labels()).tolist()) == set(range(c.n_clusters()))


def test_louvain_mode_karate_against_the_oracle():
    edges, _ = karate()
    src = np.array([a for a, _, _ in edges], np.uint64)
    dst = np.array([b for _, b, _ in edges], np.uint64)
    w = np.array([x for _, _, x in edges], np.float64)
    og = O.Graph.from_edges(34, src=src, dst=dst, w=w)
    gg = sc_gpu.CSRNetwork.from_edge_arrays(34, src, dst, w)
    for seed in range(5):
        lab_o, _ = og.leiden(seed=seed, refine=False)
        c = sc_gpu.leiden(gg, sc_gpu.LeidenConfig(seed=seed, refine=False))
        assert sc_gpu.modularity(gg, c.labels()) >= og.modularity(lab_o) - 1e-3


@pytest.mark.parametrize("cap", [60.0, 400.0])
@pytest.mark.parametrize("refine", [True, False])
def test_max_community_weight_against_the_oracle(cap, refine):
    """max_community_weight (leiden/mod.rs:80-89): no community's node weight
    passes the cap, and the quality reached under the cap is within 1e-3 of the
    oracle's under the same cap."""
    og, gg = _planted()
    lab_o, _ = og.leiden(seed=42, refine=refine, max_community_weight=cap)
    c = sc_gpu.leiden(gg, sc_gpu.LeidenConfig(seed=42, refine=refine, max_community_weight=cap))
    assert max(c.cluster_sizes()) <= cap
    assert max(np.bincount(lab_o.astype(np.int64))) <= cap
    assert sc_gpu.modularity(gg, c.labels()) >= og.modularity(lab_o) - 1e-3
