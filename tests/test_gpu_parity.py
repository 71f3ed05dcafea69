"""GPU vs oracle, bit for bit, given the same inputs and the same partition.

Covers CSRNetwork construction (from_edges, from_csr_parts, from_csr_matrix),
aggregate, Partition::from_membership aggregates, RB / CPM quality and
modularity, validate_symmetry and the error contract. Every comparison of a
float is on its bit pattern: the bar for these functions is bit-exact.
"""
import numpy as np
import pytest

import oracle as O
import sc_gpu
from sc_gpu import synth
from helpers import edges_to_arrays, karate, leidenalg_fixture, random_graph, reference_graphs

pytestmark = pytest.mark.gpu


def bits(x):
    return np.asarray(x, dtype=np.float64).view(np.uint64)


def same_f64(a, b):
    return np.array_equal(bits(a), bits(b))


def build_pair(n, edges, node_weights=None):
    src, dst, w = edges_to_arrays(edges)
    og = O.Graph.from_edges(n, src=src, dst=dst, w=w, node_weights=node_weights)
    gg = sc_gpu.CSRNetwork.from_edge_arrays(n, src, dst, w, node_weights)
    return og, gg


def assert_same_graph(og, gg, what=""):
    a = og.arrays()
    ptr, nbr, w = gg.to_csr_parts()
    assert np.array_equal(a["ptr"], ptr), what
    assert np.array_equal(a["nbr"], nbr), what
    assert np.array_equal(a["w"].view(np.uint32), w.view(np.uint32)), what
    assert same_f64(a["node_w"], gg.node_weights()), what
    assert same_f64(a["strength"], gg.strengths()), what
    assert same_f64([a["total_weight"]], [gg.total_weight()]), what
    assert a["edge_count"] == gg.edge_count(), what
    assert a["any_self_loops"] == gg.has_self_loops(), what


def odd_weight_graphs():
    """Inputs outside the exact-summation regime and with duplicate/zero entries."""
    rng = np.random.Generator(np.random.PCG64(17))
    out = []
    n = 300
    m = 4000
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    # weights spanning 60 binades: f64 sums of them round, so order matters
    w = np.exp(rng.uniform(-40, 40, m))
    out.append(("wide_range", n, list(zip(src.tolist(), dst.tolist(), w.tolist()))))
    w2 = np.where(rng.random(m) < 0.5, 1e-14, 1.0) * rng.uniform(0.5, 1.5, m)
    out.append(("tiny_and_unit", n, list(zip(src.tolist(), dst.tolist(), w2.tolist()))))
    dup = [(0, 1, 0.1), (1, 0, 0.2), (0, 1, 0.3), (2, 2, 0.7), (2, 2, 0.9), (3, 4, 0.0), (4, 3, 0.0),
           (5, 6, 1e30), (5, 6, 1.0), (6, 5, -0.0)]
    out.append(("duplicates_and_zeros", 8, dup))
    return out


def all_graphs():
    gs = [(name, n, e) for name, n, e in reference_graphs()]
    for seed in range(12):
        n, e = random_graph(seed)
        gs.append((f"random{seed}", n, e))
    gs += odd_weight_graphs()
    return gs


@pytest.mark.parametrize("name,n,edges", all_graphs(), ids=lambda x: x if isinstance(x, str) else "")
def test_from_edges_bit_exact(name, n, edges):
    og, gg = build_pair(n, edges)
    assert_same_graph(og, gg, name)


def test_from_edges_planted_partition_20k():
    src, dst, w, _ = synth.planted_partition()
    og = O.Graph.from_edges(20000, src=src, dst=dst, w=w)
    gg = sc_gpu.CSRNetwork.from_edge_arrays(20000, src, dst, w)
    assert_same_graph(og, gg, "C1")


def test_from_edges_with_node_weights():
    rng = np.random.Generator(np.random.PCG64(5))
    n, edges = random_graph(3)
    nw = rng.uniform(0.1, 5.0, n)
    og, gg = build_pair(n, edges, nw)
    assert_same_graph(og, gg)


def _shuffled_csr(og, seed, dup=False):
    a = og.arrays()
    rng = np.random.Generator(np.random.PCG64(seed))
    ptr, nbr, w = a["ptr"], a["nbr"].copy(), a["w"].copy()
    rows_n, rows_w = [], []
    for v in range(a["n"]):
        s, e = int(ptr[v]), int(ptr[v + 1])
        idx = rng.permutation(e - s)
        rn, rw = list(nbr[s:e][idx]), list(w[s:e][idx])
        if dup and e > s:
            # split one weight in two parts (both parts exactly representable)
            rn.append(rn[0])
            half = np.float32(rw[0]) / np.float32(2)
            rw[0] = half
            rw.append(half)
            rn.append(rn[0])
            rw.append(np.float32(0.0))
        rows_n.append(rn)
        rows_w.append(rw)
    nptr = np.zeros(a["n"] + 1, np.uint64)
    nptr[1:] = np.cumsum([len(r) for r in rows_n])
    flat_n = np.array([x for r in rows_n for x in r], np.uint32)
    flat_w = np.array([x for r in rows_w for x in r], np.float32)
    return nptr, flat_n, flat_w


@pytest.mark.parametrize("dup", [False, True])
def test_from_csr_parts_bit_exact(dup):
    for name, n, edges in all_graphs():
        src, dst, w = edges_to_arrays(edges)
        base = O.Graph.from_edges(n, src=src, dst=dst, w=w)
        ptr, nbr, ww = _shuffled_csr(base, 7, dup)
        if n == 0:
            ptr = np.zeros(1, np.uint64)
        og = O.Graph.from_csr_parts(ptr, nbr, ww)
        gg = sc_gpu.CSRNetwork.from_csr_parts(ptr, nbr, ww)
        assert_same_graph(og, gg, name)


def test_from_csr_matrix_reads_upper_triangle():
    rng = np.random.Generator(np.random.PCG64(9))
    n = 50
    dense = np.triu(rng.random((n, n)) * (rng.random((n, n)) < 0.2))
    dense = dense + np.triu(dense, 1).T
    # the lower triangle is ignored: make it garbage
    dense[np.tril_indices(n, -1)] *= 3.0
    indptr = np.zeros(n + 1, np.uint64)
    indices, data = [], []
    for r in range(n):
        cols = np.nonzero(dense[r])[0]
        indices += cols.tolist()
        data += dense[r, cols].tolist()
        indptr[r + 1] = len(indices)
    og = O.Graph.from_csr_matrix(indptr, indices, data)
    gg = sc_gpu.CSRNetwork.from_csr_matrix(indptr, indices, data)
    assert_same_graph(og, gg)


def partitions_for(n, seed, og):
    rng = np.random.Generator(np.random.PCG64(seed))
    ps = [np.arange(n, dtype=np.uint64), np.zeros(n, np.uint64)]
    if n:
        ps.append(rng.integers(0, max(1, n // 3), n).astype(np.uint64))
        ps.append((rng.integers(0, 4, n) * 1000 + 7).astype(np.uint64))  # sparse slot ids
        lab, _ = og.leiden(seed=seed)
        ps.append(lab)
    return ps


@pytest.mark.parametrize("name,n,edges", all_graphs(), ids=lambda x: x if isinstance(x, str) else "")
def test_aggregate_bit_exact(name, n, edges):
    og, gg = build_pair(n, edges)
    for i, p in enumerate(partitions_for(n, 3, og)):
        assert_same_graph(og.aggregate(p), gg.aggregate(p), f"{name} partition {i}")


@pytest.mark.parametrize("name,n,edges", all_graphs(), ids=lambda x: x if isinstance(x, str) else "")
def test_quality_and_modularity_bit_exact(name, n, edges):
    og, gg = build_pair(n, edges)
    for i, p in enumerate(partitions_for(n, 5, og)):
        for obj, res in ((O.RB, 1.0), (O.RB, 0.37), (O.CPM, 0.05), (O.CPM, 1.0)):
            kind = sc_gpu.Rb(res) if obj == O.RB else sc_gpu.Cpm(res)
            assert same_f64([og.quality(p, obj, res)], [sc_gpu.quality(gg, p, kind)]), (name, i, obj, res)
        for gamma in (1.0, 0.5, 2.0):
            assert same_f64([og.modularity(p, gamma)], [sc_gpu.modularity(gg, p, gamma)]), (name, i, gamma)
        so, sg = og.partition_stats(p), gg.partition_stats(p)
        assert np.array_equal(so["size"], sg["size"])
        for k in ("weight", "strength", "internal"):
            assert same_f64(so[k], sg[k]), (name, i, k)


def test_aggregate_planted_partition_20k():
    src, dst, w, truth = synth.planted_partition()
    og = O.Graph.from_edges(20000, src=src, dst=dst, w=w)
    gg = sc_gpu.CSRNetwork.from_edge_arrays(20000, src, dst, w)
    lab, _ = og.leiden(seed=42)
    for p in (lab, truth, np.arange(20000, dtype=np.uint64) // 7):
        assert_same_graph(og.aggregate(p), gg.aggregate(p))
        assert same_f64([og.modularity(p)], [sc_gpu.modularity(gg, p)])
        assert same_f64([og.quality(p)], [sc_gpu.quality(gg, p)])


def test_aggregate_of_balanced_asymmetric_graph():
    """A graph whose degree sums balance but whose rows do not mirror
    (csr_network.rs:968-979) takes the ordered sort path of aggregate; a
    symmetric one in the exact regime takes the per-row hash contraction. Both
    must give the reference's bits."""
    ptrs, nbrs, ws = [0, 2, 3, 4], [1, 2, 0, 0], [1.0, 3.0, 3.0, 1.0]
    og = O.Graph.from_csr_parts(np.array(ptrs, np.uint64), np.array(nbrs, np.uint32), np.array(ws, np.float32))
    gg = sc_gpu.CSRNetwork.from_csr_parts(ptrs, nbrs, ws)
    for p in ([0, 0, 1], [0, 1, 1], [0, 1, 2], [0, 0, 0]):
        assert_same_graph(og.aggregate(np.array(p, np.uint64)), gg.aggregate(p))


def test_aggregate_large_rows_use_the_block_contraction():
    """Each row-size path of the exact-regime contraction: small rows (a warp
    per row), one large row whose table fits shared memory, one large row with
    more distinct neighbour groups than that (its entries sorted as (g, h) keys
    and summed per segment), and large rows holding most entries (the sort path
    of the whole graph, with segments long enough for the chunked sums)."""
    src, dst, w, truth = synth.planted_partition(6000, 6, 12, 3, seed=4)
    og = O.Graph.from_edges(6000, src=src, dst=dst, w=w)
    gg = sc_gpu.CSRNetwork.from_edge_arrays(6000, src, dst, w)
    v = np.arange(6000)
    shared_row = np.where(v < 300, 0, 1 + (v - 300) // 3).astype(np.uint64)
    global_row = np.where(v < 200, 0, v - 199).astype(np.uint64)
    for p in (shared_row, global_row, truth, np.zeros(6000, np.uint64)):
        assert_same_graph(og.aggregate(p), gg.aggregate(p))


def test_leidenalg_fixture_definitions():
    # tests/reference.rs:164-209 on the GPU quality and modularity
    d = leidenalg_fixture()
    graphs = {k: sc_gpu.CSRNetwork.from_edges(v["n_nodes"], [tuple(e) for e in v["edges"]])
              for k, v in d["graphs"].items()}
    for c in d["cases"]:
        g = graphs[c["graph"]]
        kind = sc_gpu.Rb(c["resolution"]) if c["objective"] == "rb" else sc_gpu.Cpm(c["resolution"])
        q = sc_gpu.quality(g, c["reference_membership"], kind) * 2
        assert abs(q - c["reference_quality"]) <= 1e-6 * max(abs(c["reference_quality"]), 1.0)
        m = sc_gpu.modularity(g, c["reference_membership"], 1.0)
        assert abs(m - c["reference_modularity"]) <= 1e-7


def test_validate_symmetry():
    # csr_network.rs:955-979
    og, gg = build_pair(6, [(0, 1, 2.5), (2, 3, 0.5), (4, 4, 1.0)])
    gg.validate_symmetry()
    bad = sc_gpu.CSRNetwork.from_csr_parts([0, 2, 3, 4], [1, 2, 0, 0], [1.0, 3.0, 3.0, 1.0])
    with pytest.raises(sc_gpu.InvalidCsr):
        bad.validate_symmetry()


ERROR_CASES = [
    ("csr", ([0, 5], [0], [1.0]), sc_gpu.InvalidCsr),
    ("csr", ([0, 1], [0], [1.0, 2.0]), sc_gpu.InvalidCsr),
    ("csr", ([0, 1], [9], [1.0]), sc_gpu.NodeIndexOutOfRange),
    ("csr", ([0, 2, 1], [0, 1], [1.0, 1.0]), sc_gpu.InvalidCsr),
    ("csr", ([], [], []), sc_gpu.InvalidCsr),
    ("csr", ([0, 1, 1], [1], [1.0]), sc_gpu.AsymmetricGraph),
    ("csr", ([0, 1, 2], [1, 0], [1.0, 5.0]), sc_gpu.AsymmetricGraph),
    ("csr", ([0, 1, 2], [1, 0], [1.0, float("inf")]), sc_gpu.NonFiniteWeight),
    ("csr", ([0, 1, 2], [1, 0], [-1.0, -1.0]), sc_gpu.NegativeWeight),
    ("edges", (2, [(0, 5, 1.0)]), sc_gpu.NodeIndexOutOfRange),
    ("edges", (2, [(0, 1, -1.0)]), sc_gpu.NegativeWeight),
    ("edges", (2, [(0, 1, float("nan"))]), sc_gpu.NonFiniteWeight),
]


@pytest.mark.parametrize("kind,args,exc", ERROR_CASES)
def test_errors_match_the_reference(kind, args, exc):
    with pytest.raises(O.OracleError) as oe:
        if kind == "csr":
            O.Graph.from_csr_parts(*args)
        else:
            O.Graph.from_edges(*args)
    with pytest.raises(exc) as ge:
        if kind == "csr":
            sc_gpu.CSRNetwork.from_csr_parts(*args)
        else:
            sc_gpu.CSRNetwork.from_edges(*args)
    assert ge.value.status == oe.value.code
    gi, oi = ge.value.info, oe.value.info
    for f in ("node", "n_nodes", "edge_from", "edge_to", "got", "expected_len"):
        assert getattr(gi, f) == getattr(oi, f), f
    for f in ("weight", "degree_sum", "expected"):
        assert same_f64([getattr(gi, f)], [getattr(oi, f)]), f


def test_node_weight_errors():
    with pytest.raises(sc_gpu.NodeWeightLengthMismatch):
        sc_gpu.CSRNetwork.from_csr_parts([0, 1, 2], [1, 0], [1.0, 1.0], [1.0])
    with pytest.raises(sc_gpu.InvalidNodeWeight) as e:
        sc_gpu.CSRNetwork.from_csr_parts([0, 1, 2], [1, 0], [1.0, 1.0], [1.0, -2.0])
    assert e.value.node == 1 and e.value.weight == -2.0
    with pytest.raises(sc_gpu.MembershipLengthMismatch):
        g = sc_gpu.CSRNetwork.from_edges(3, [(0, 1, 1.0)])
        sc_gpu.modularity(g, [0, 1])
