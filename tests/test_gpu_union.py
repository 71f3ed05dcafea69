"""Batched runs over a disjoint union of instances (sc_leiden_batch_union).

Every kernel launch covers the nodes of all instances; each node reads its
instance's resolution, seed and totals, hashes instance-local ids, and an
instance stops where its own run stops. Inside the exact summation regime
(all graphs here) every instance's labels must equal those of its own
leiden() / leiden_from() call bit for bit (src/community_search/leiden/mod.rs:168-220).
"""
import numpy as np
import pytest

import sc_gpu
from sc_gpu import synth
from helpers import reference_graphs, edges_to_arrays

pytestmark = pytest.mark.gpu


def _graph(n, edges):
    src, dst, w = edges_to_arrays(edges)
    return sc_gpu.CSRNetwork.from_edge_arrays(n, src, dst, w)


def _planted_set(count=40, seed=5):
    out = []
    for n, src, dst, w, _ in synth.many_planted_graphs(count, seed, n_range=(30, 4000)):
        out.append(sc_gpu.CSRNetwork.from_edge_arrays(n, src, dst, w))
    return out


def _separate(graphs, cfgs, warm_from=None):
    labels, ncl = [], []
    for i, (g, c) in enumerate(zip(graphs, cfgs)):
        if warm_from is not None and warm_from[i] >= 0:
            r = sc_gpu.leiden_from(g, c, labels[warm_from[i]])
        else:
            r = sc_gpu.leiden(g, c)
        labels.append(r.labels())
        ncl.append(r.n_clusters())
    return labels, ncl


def _assert_same(batch, labels, ncl):
    assert len(batch) == len(labels)
    for i, (b, l, k) in enumerate(zip(batch, labels, ncl)):
        assert b.n_clusters() == k, i
        assert np.array_equal(b.labels(), l), i


@pytest.mark.parametrize("objective", [sc_gpu.Rb, sc_gpu.Cpm])
def test_union_equals_separate_runs_on_uneven_graphs(objective):
    graphs = _planted_set()
    graphs += [_graph(n, e) for _, n, e in reference_graphs()]  # empty, single node, no edges, loops, ...
    rng = np.random.default_rng(3)
    gam = (lambda: float(rng.uniform(0.3, 3.0))) if objective is sc_gpu.Rb else (lambda: float(rng.uniform(0.02, 0.3)))
    cfgs = [sc_gpu.LeidenConfig(objective=objective(gam()), seed=int(rng.integers(1, 1 << 30)))
            for _ in graphs]
    labels, ncl = _separate(graphs, cfgs)
    _assert_same(sc_gpu.leiden_batch(graphs, cfgs, union=True), labels, ncl)
    # a small entry cap splits the instances over several unions
    _assert_same(sc_gpu.leiden_batch(graphs, cfgs, union=True, max_union_entries=20000), labels, ncl)


def test_union_equals_separate_runs_with_options():
    graphs = _planted_set(16, 9)
    for extra in ({"refine": False}, {"max_community_weight": 40.0}, {"n_iterations": 4, "patience": 1},
                  {"max_levels": 2}, {"refine_randomness": 0.0}):
        cfgs = [sc_gpu.LeidenConfig(objective=sc_gpu.Rb(0.5 + 0.1 * i), seed=100 + i, **extra)
                for i in range(len(graphs))]
        labels, ncl = _separate(graphs, cfgs)
        _assert_same(sc_gpu.leiden_batch(graphs, cfgs, union=True), labels, ncl)


def test_union_sweep_with_warm_chains_equals_separate_runs():
    X, _ = synth.gaussian_mixture(20000, 30, 20, 4, sigma=(0.7, 1.5))
    r = sc_gpu.knn_gaussian(X, 10, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION)
    g = sc_gpu.CSRNetwork.from_csr_parts(r.conn_ptrs, r.conn_nbrs, r.conn_w)
    res = np.geomspace(0.2, 3.0, 8)
    cfgs, warm, keys = sc_gpu.sweep_plan(res, [1, 2], split=2)
    labels, ncl = _separate([g] * len(cfgs), cfgs, warm)
    out = sc_gpu.leiden_batch([g] * len(cfgs), cfgs, warm, union=True)
    _assert_same(out, labels, ncl)
    sw = sc_gpu.leiden_sweep(g, res, [1, 2], split=2, union=True)
    for k, lab in zip(keys, labels):
        assert np.array_equal(sw[k].labels(), lab)


def test_union_rejects_mixed_objectives():
    graphs = _planted_set(3, 2)
    cfgs = [sc_gpu.LeidenConfig(objective=sc_gpu.Rb(1.0)), sc_gpu.LeidenConfig(objective=sc_gpu.Cpm(0.1)),
            sc_gpu.LeidenConfig()]
    with pytest.raises(sc_gpu.InvalidConfig):
        sc_gpu.leiden_batch(graphs, cfgs, union=True)
    # the context stays usable
    assert sc_gpu.leiden(graphs[0]).n_clusters() >= 1
