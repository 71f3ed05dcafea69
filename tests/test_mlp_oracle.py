"""CPU checks of the learned-warm-start oracle (oracle/mlp_oracle.py).

The GPU kernels are compared against this oracle in test_gpu_mlp.py; here the
oracle itself is pinned: its analytic gradient against central finite
differences, its BF16 rounding against known bit patterns, its features and
components against hand-worked graphs.
"""
import numpy as np
import pytest

import mlp_oracle as mo


def _rand_params(rng, scale=0.3):
    return rng.normal(0.0, scale, mo.n_params())


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    X = rng.normal(size=(40, mo.F))
    y = (rng.random(40) < 0.6).astype(np.float64)
    p = _rand_params(rng)
    loss, g = mo.forward_backward(p, X, y)
    eps = 1e-6
    idx = rng.choice(mo.n_params(), 60, replace=False)
    idx = np.concatenate([idx, [mo.n_params() - 1]])  # b2 too
    for i in idx:
        d = np.zeros_like(p)
        d[i] = eps
        lp, _ = mo.forward_backward(p + d, X, y)
        lm, _ = mo.forward_backward(p - d, X, y)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    assert loss > 0


def test_bce_matches_direct_formula():
    rng = np.random.default_rng(1)
    X = rng.normal(size=(25, mo.F))
    y = (rng.random(25) < 0.5).astype(np.float64)
    p = _rand_params(rng)
    loss, _ = mo.forward_backward(p, X, y)
    q = mo.probabilities(p, X)
    direct = -np.mean(y * np.log(q) + (1 - y) * np.log(1 - q))
    assert abs(loss - direct) < 1e-12


def test_bf16_rounding_known_values():
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.001953125, -2.5, 3.0e38, 0.0, 1.01171875], np.float32)
    got = mo.bf16_round(vals)
    # BF16 keeps 7 fraction bits: next above 1 is 1 + 2^-7. 1 + 2^-8 is a tie
    # -> even (1.0); 1 + 1.5*2^-8 rounds up; 1 + 2^-9 rounds down;
    # 1 + 3*2^-8 is a tie between 1 + 2^-7 (odd) and 1 + 2^-6 (even) -> up
    assert got[0] == 1.0 and got[1] == 1.0
    assert got[2] == np.float32(1.0078125) and got[3] == 1.0
    assert got[7] == np.float32(1.015625)
    assert got[4] == -2.5 and got[6] == 0.0
    assert (got.view(np.uint32) & 0xFFFF).max() == 0


def test_features_on_triangle_with_tail():
    # 0-1-2 triangle (weights 1, 2, 3) plus the tail 2-3 (weight 1)
    ptr = np.array([0, 2, 4, 7, 8])
    nbr = np.array([1, 2, 0, 2, 0, 1, 3, 2])
    w = np.array([1, 3, 1, 2, 3, 2, 1, 1], np.float32)
    strength = np.array([4.0, 3.0, 6.0, 1.0])
    feats, ei, ej = mo.edge_features(ptr, nbr, w, strength, 7.0, 1.0)
    assert list(zip(ei, ej)) == [(0, 1), (0, 2), (1, 2), (2, 3)]
    f01 = feats[0]
    assert f01[0] == 1.0
    assert np.isclose(f01[7], 1.0 * 4.0 * 3.0 / (14.0 * 1.0))
    # common neighbour of (0, 1) is 2 with min(w02, w12) = min(3, 2) = 2; min strength 3
    assert np.isclose(f01[8], 2.0 / 3.0) and np.isclose(f01[9], 1.0 / 2.0)
    # the tail edge has no common neighbour
    assert feats[3][8] == 0.0 and feats[3][9] == 0.0
    assert np.allclose(feats[:, mo.GAMMA_FEATURE], 0.0)
    assert np.all(feats[:, 10:] == 0.0)  # no context partitions
    feats2, _, _ = mo.edge_features(ptr, nbr, w, strength, 7.0, 1.0, coarse=[0, 0, 0, 1], fine=[0, 1, 1, 2])
    # edges (0,1) (0,2) (1,2) (2,3): together at coarse 1 1 1 0, at fine 0 0 1 0
    assert list(feats2[:, 10]) == [1, 1, 1, 0] and list(feats2[:, 11]) == [0, 0, 1, 0]
    # neighbour-label histograms read at the other endpoint's community:
    # (0,1) coarse: 0 sends 4/4 and 1 sends 3/3 of its strength to label 0 -> 1;
    # (2,3) coarse: 2 sends 1/6 to label 1, 3 sends 1/1 to label 0 -> 7/12;
    # (0,1) fine: 0 sends 4/4 to label 1, 1 sends 1/3 to label 0 -> 2/3
    assert np.isclose(feats2[0, 12], 1.0) and np.isclose(feats2[3, 12], 7.0 / 12.0)
    assert np.isclose(feats2[0, 13], 2.0 / 3.0)
    assert np.all(feats2[:, 14] == 0.0)  # no embedding


def test_embedding_feature_is_scale_and_shift_free():
    # triangle with a tail again; points in 5-D
    ptr = np.array([0, 2, 4, 7, 8])
    nbr = np.array([1, 2, 0, 2, 0, 1, 3, 2])
    w = np.array([1, 3, 1, 2, 3, 2, 1, 1], np.float32)
    strength = np.array([4.0, 3.0, 6.0, 1.0])
    X = np.random.default_rng(3).normal(size=(4, 5))
    f1, _, _ = mo.edge_features(ptr, nbr, w, strength, 7.0, 1.0, embedding=X)
    f2, _, _ = mo.edge_features(ptr, nbr, w, strength, 7.0, 1.0, embedding=3.0 * X + 5.0)
    assert np.all(f1[:, 14] > 0.0)
    assert np.allclose(f1[:, 14], f2[:, 14], rtol=1e-12)
    assert np.array_equal(f1[:, :14], f2[:, :14])
    P = mo.projection(5)
    assert P.shape == (5, mo.EMB_R) and set(np.unique(P)) <= {-0.25, 0.25}
    # edge (0, 1) by hand: its projected length over the endpoints' mean scale
    y = X @ P
    s0 = np.mean([np.sum((y[0] - y[v]) ** 2) for v in (1, 2)])
    s1 = np.mean([np.sum((y[1] - y[v]) ** 2) for v in (0, 2)])
    assert np.isclose(f1[0, 14], np.sum((y[0] - y[1]) ** 2) / (0.5 * (s0 + s1)))


def test_scaler_passes_gamma_through():
    rng = np.random.default_rng(0)
    raw = rng.normal(2.0, 3.0, size=(500, mo.F))
    raw[:, mo.GAMMA_FEATURE] = np.log(0.5)
    mean, istd = mo.scaler_fit(raw)
    assert mean[mo.GAMMA_FEATURE] == 0.0 and istd[mo.GAMMA_FEATURE] == 1.0
    z = (raw - mean) * istd
    keep = [f for f in range(mo.F) if f != mo.GAMMA_FEATURE]
    assert np.allclose(z[:, keep].mean(axis=0), 0.0, atol=1e-12)
    assert np.allclose(z[:, keep].std(axis=0), 1.0, atol=1e-9)


def test_components_numbered_by_smallest_member():
    ei = np.array([0, 1, 3, 4, 2])
    ej = np.array([5, 5, 6, 6, 7])
    mask = np.array([True, True, True, False, False])
    lab = mo.components(8, ei, ej, mask)
    # {0,1,5} {2} {3,6} {4} {7}
    assert list(lab) == [0, 0, 1, 2, 3, 0, 2, 4]


@pytest.mark.parametrize("M", [0, 1])
def test_tiny_edge_sets(M):
    p = np.zeros(mo.n_params())
    X = np.zeros((M, mo.F))
    y = np.ones(M)
    loss, g = mo.forward_backward(p, X, y)
    assert g.shape == (mo.n_params(),)
    if M:
        assert np.isclose(loss, np.log(2.0))
