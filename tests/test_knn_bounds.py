"""CPU checks of the score bound the pruned kNN search's second pass starts
from (k_pass2_cap in single-clustering_b200/csrc/sc_knn.cu).

The tensor-core score of query x and point y is sum_j bf16(-2 bf16(x_j)) bf16(y_j)
+ hi + lo (hi + lo the two-BF16 split of |y|^2), accumulated in FP32. The cap
assumes it lies within 2^-6 (1 + 2^-6) |x| Y + 2^-14 Y^2 of |y|^2 - 2 x.y for
|y| <= Y: the input roundings' bound (4u + 2u^2) |x| |y| with u = 2^-8, plus
room for the norm split and the FP32 accumulation.
Here the roundings are reproduced in numpy (products and sums in FP64, so the
accumulation term of the bound is left as slack) on random and adversarial
vectors (every coordinate just below a BF16 rounding midpoint, the same sign
throughout: the worst case of the input roundings, which comes within a few
percent of the bound), and the bound must hold.
"""
import numpy as np

import mlp_oracle as mo


def _score_bf16(x, y):
    xb = mo.bf16_round(x).astype(np.float64)
    yb = mo.bf16_round(y).astype(np.float64)
    a = mo.bf16_round((-2.0 * xb).astype(np.float32)).astype(np.float64)
    nrm = np.float32(0.0)
    for t in y.astype(np.float32):
        nrm = np.float32(nrm + np.float32(t * t))  # FP32 norm (the kernel fuses; either is within the slack)
    hi = mo.bf16_round(np.array([nrm], np.float32)).astype(np.float64)[0]
    lo = mo.bf16_round(np.array([np.float32(nrm - np.float32(hi))], np.float32)).astype(np.float64)[0]
    return float(a @ yb + hi + lo)


def _margin(x, Y):
    nx = float(np.linalg.norm(x.astype(np.float64)))
    return 2.0 ** -6 * (1 + 2.0 ** -6) * nx * Y + 2.0 ** -14 * Y * Y


def test_bf16_score_error_within_the_cap_margin():
    rng = np.random.Generator(np.random.PCG64(7))
    worst = 0.0
    for trial in range(3000):
        d = int(rng.integers(1, 63))
        scale = float(10.0 ** rng.uniform(-3, 3))
        kind = trial % 3
        if kind == 0:    # isotropic
            x = rng.normal(size=d) * scale
            y = x + rng.normal(size=d) * scale * rng.uniform(0.01, 1.0)
        elif kind == 1:  # every coordinate the same sign (no cancellation in x.y)
            x = np.abs(rng.normal(size=d)) * scale
            y = np.abs(rng.normal(size=d)) * scale
        else:            # coordinates just below BF16 rounding midpoints, one sign
            p2 = 2.0 ** int(rng.integers(-10, 10))
            x = np.full(d, (1.0 + 2.0 ** -8 * (1 - 2.0 ** -10)) * p2)
            y = np.full(d, (1.0 + 2.0 ** -8 * (1 - 2.0 ** -10)) * p2)
        x = x.astype(np.float32)
        y = y.astype(np.float32)
        exact = float(y.astype(np.float64) @ y.astype(np.float64) - 2.0 * (x.astype(np.float64) @ y.astype(np.float64)))
        err = abs(_score_bf16(x, y) - exact)
        Y = float(np.linalg.norm(y.astype(np.float64)))
        m = _margin(x, Y)
        assert err <= m, (trial, d, err, m)
        worst = max(worst, err / m)
    # the worst case of the roundings reaches the input-rounding bound: the
    # margin is tight, with the rest covering the norm and the accumulation
    assert 0.9 < worst <= 1.0, worst
