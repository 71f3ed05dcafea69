"""The seeded synthetic workloads: same bytes for the same seed, and the
shapes the benchmark configurations name (checked on the CPU)."""
import numpy as np
import pytest

from sc_gpu import synth


def test_planted_partition_is_seeded_and_planted():
    a = synth.planted_partition(2000, 10, 6, 2, seed=3)
    b = synth.planted_partition(2000, 10, 6, 2, seed=3)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    src, dst, w, truth = a
    assert len(src) == 2000 * (6 + 2)
    intra = truth[src.astype(np.int64)] == truth[dst.astype(np.int64)]
    assert intra.sum() == 2000 * 6  # the intra draws stay inside the block, the others leave it
    assert np.all(src != dst)
    assert w.min() >= 0.5 and w.max() <= 1.5 and np.array_equal(w, w.astype(np.float32))


def test_many_planted_graphs_shapes():
    graphs = list(synth.many_planted_graphs(64, seed=21))
    again = list(synth.many_planted_graphs(64, seed=21))
    assert len(graphs) == 64
    ns = np.array([g[0] for g in graphs])
    assert ns.min() >= 100 and ns.max() <= 50_000
    for (n, src, dst, w, truth), (n2, src2, dst2, w2, truth2) in zip(graphs, again):
        assert n == n2 and np.array_equal(src, src2) and np.array_equal(dst, dst2) and np.array_equal(w, w2)
        blocks = int(truth.max()) + 1
        assert 1 <= blocks <= max(1, n // 5)
        mean_degree = 2.0 * len(src) / n
        assert 9.0 <= mean_degree <= 31.0
        share = np.mean(truth[src.astype(np.int64)] == truth[dst.astype(np.int64)])
        assert 0.6 <= share <= 1.0


def test_gaussian_mixture_is_seeded():
    x1, c1 = synth.gaussian_mixture(5000, 7, 4, seed=9, sigma=(0.5, 1.0))
    x2, c2 = synth.gaussian_mixture(5000, 7, 4, seed=9, sigma=(0.5, 1.0))
    assert x1.dtype == np.float32 and x1.shape == (5000, 7)
    assert np.array_equal(x1, x2) and np.array_equal(c1, c2)
    assert set(np.unique(c1)) <= set(range(4))


@pytest.mark.parametrize("n,d,comps,k", [(4000, 30, 10, 10), (2500, 50, 3, 15), (300, 7, 40, 5)])
def test_exact_torch_knn_graph_matches_the_fp64_oracle(n, d, comps, k):
    """The benchmark's library-free input builder: its k+1 lists equal the FP64
    oracle's (pruning by ball bounds is exact for any grouping), and its graph is
    the oracle's union-symmetrised Gaussian connectivities (sigma = k-th
    distance) rounded to f32."""
    import knn_oracle as K
    X, comp = synth.gaussian_mixture(n, d, comps, seed=n + d, sigma=(0.7, 1.5))
    it, dt = K.knn_exact(X, k)
    for groups in (comp, np.random.default_rng(0).integers(0, 7, n)):
        ptr, nbr, w, idx, dist = synth.knn_graph_exact_torch(X, groups, k, "cpu", chunk=700)
        assert np.array_equal(idx, it)
        assert np.abs(dist - dt).max() < 1e-12
    r, c, ww = K.connectivities(it, dt, K.sigmas(dt, kth=True), union=True)
    rows = np.repeat(np.arange(n), np.diff(ptr).astype(np.int64))
    assert np.array_equal(rows, r) and np.array_equal(nbr, c)
    assert np.array_equal(w, ww.astype(np.float32))
