"""CPU oracle of the learned warm start (test infrastructure only).

The product computes these on the GPU (single-clustering_b200/csrc/sc_mlp.cu);
tests compare against this numpy FP64 restatement:

* edge_features: the raw (unscaled) features of every undirected edge i < j of
  a CSR graph, in ascending (i, j) order;
* forward_backward: mean binary cross-entropy of the 2-layer MLP and its
  gradient, evaluated with BF16-rounded weights (the GPU's forward weights) in
  FP64, so the GPU's FP32-accumulated gradient can be checked against it;
* core_mask, components: the edges the proposal keeps (confident, between
  core nodes) and their connected components, numbered by smallest member.

single-clustering itself has no learned part; what this pins is the GPU's
arithmetic, and finite differences pin this oracle's own gradient.
"""
from __future__ import annotations

import numpy as np

F = 15
EMB_R = 16
H = 128
GAMMA_FEATURE = 6


def n_params() -> int:
    return F * H + H + H + 1


def bf16_round(x) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def unpack(params):
    p = np.asarray(params, np.float64)
    W1 = p[:F * H].reshape(F, H)
    b1 = p[F * H:F * H + H]
    w2 = p[F * H + H:F * H + 2 * H]
    b2 = p[F * H + 2 * H]
    return W1, b1, w2, b2


def _splitmix(x: int) -> int:
    m = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & m
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    return x ^ (x >> 31)


def projection(d: int) -> np.ndarray:
    """The d x EMB_R sign matrix of the embedding feature: +-1/4, negative where
    the top bit of splitmix64(a * EMB_R + r) is set."""
    P = np.empty((d, EMB_R), np.float64)
    for a in range(d):
        for r in range(EMB_R):
            P[a, r] = -0.25 if _splitmix(a * EMB_R + r) >> 63 else 0.25
    return P


def edge_features(ptr, nbr, w, strength, total_weight, gamma, coarse=None, fine=None, embedding=None):
    """Raw features of the undirected edges (sc_mlp.cu k_edge_features);
    coarse / fine: labels of the neighbouring-resolution partitions or None;
    embedding: the n x d points the graph was built from, or None."""
    ptr = np.asarray(ptr, np.int64)
    nbr = np.asarray(nbr, np.int64)
    w = np.asarray(w, np.float32)
    n = len(ptr) - 1
    rows = [set() for _ in range(n)]
    wmap = [dict() for _ in range(n)]
    for i in range(n):
        for x in range(ptr[i], ptr[i + 1]):
            rows[i].add(int(nbr[x]))
            wmap[i][int(nbr[x])] = float(w[x])
    ei, ej, feats = [], [], []
    two_m = 2.0 * total_weight
    y = scale = None
    if embedding is not None:
        X = np.asarray(embedding, np.float64)
        y = X @ projection(X.shape[1])
        scale = np.zeros(n)
        for i in range(n):
            nb = [int(v) for v in nbr[ptr[i]:ptr[i + 1]] if int(v) != i]
            scale[i] = np.mean([np.sum((y[i] - y[v]) ** 2) for v in nb]) if nb else 0.0

    memo = {}

    def share(i, L, labels, ki):
        # Σ over the row in ascending neighbour order (the kernel's order);
        # memoised per (partition, node, label): hub rows are long
        key = (id(labels), i, int(L))
        if key not in memo:
            s = 0.0
            for x in range(ptr[i], ptr[i + 1]):
                v = int(nbr[x])
                if v != i and labels[v] == L:
                    s += float(w[x])
            memo[key] = s / max(ki, 1e-300)
        return memo[key]
    for i in range(n):
        for x in range(ptr[i], ptr[i + 1]):
            j = int(nbr[x])
            if not i < j:
                continue
            wij = float(w[x])
            ki, kj = float(strength[i]), float(strength[j])
            di, dj = float(ptr[i + 1] - ptr[i]), float(ptr[j + 1] - ptr[j])
            lki, lkj, ldi, ldj = np.log1p(ki), np.log1p(kj), np.log(di), np.log(dj)
            common = (rows[i] & rows[j]) - {i, j}
            cw = sum(min(np.float32(wmap[i][c]), np.float32(wmap[j][c])) for c in common)
            f = [wij, lki + lkj, abs(lki - lkj), ldi + ldj, abs(ldi - ldj),
                 wij / max(ki, 1e-300) + wij / max(kj, 1e-300), np.log(gamma),
                 gamma * ki * kj / (two_m * max(wij, 1e-300)) if two_m > 0 else 0.0,
                 cw / max(min(ki, kj), 1e-300), len(common) / max(min(di, dj), 1.0),
                 0.0 if coarse is None else float(coarse[i] == coarse[j]),
                 0.0 if fine is None else float(fine[i] == fine[j]),
                 0.0 if coarse is None else 0.5 * (share(i, coarse[j], coarse, ki) + share(j, coarse[i], coarse, kj)),
                 0.0 if fine is None else 0.5 * (share(i, fine[j], fine, ki) + share(j, fine[i], fine, kj)),
                 0.0 if y is None else float(np.sum((y[i] - y[j]) ** 2)) / max(0.5 * (scale[i] + scale[j]), 1e-30)]
            ei.append(i)
            ej.append(j)
            feats.append(f)
    return np.array(feats, np.float64).reshape(-1, F), np.array(ei, np.int64), np.array(ej, np.int64)


def scaler_fit(raw):
    """Means and inverse standard deviations (log gamma passed through)."""
    raw = np.asarray(raw, np.float64)
    mean = raw.mean(axis=0) if len(raw) else np.zeros(F)
    var = np.maximum((raw * raw).mean(axis=0) - mean * mean, 0.0) if len(raw) else np.zeros(F)
    istd = np.where(var > 1e-12, 1.0 / np.sqrt(np.maximum(var, 1e-300)), 1.0)
    mean[GAMMA_FEATURE] = 0.0
    istd[GAMMA_FEATURE] = 1.0
    return mean, istd


def forward(params, X):
    W1, b1, w2, b2 = unpack(params)
    A = X @ W1 + b1
    Hh = np.maximum(A, 0.0)
    z = Hh @ w2 + b2
    return A, Hh, z


def forward_backward(params, X, y):
    """(mean BCE loss, gradient) in FP64 at `params` (round them to BF16 first
    to mirror the GPU forward)."""
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    M = len(X)
    W1, b1, w2, b2 = unpack(params)
    A, Hh, z = forward(params, X)
    loss = np.mean(np.maximum(z, 0.0) - z * y + np.log1p(np.exp(-np.abs(z)))) if M else 0.0
    p = 1.0 / (1.0 + np.exp(-z))
    dz = (p - y) / max(M, 1)
    gw2 = Hh.T @ dz
    gb2 = dz.sum()
    dA = np.outer(dz, w2) * (A > 0)
    gW1 = X.T @ dA
    gb1 = dA.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gw2, [gb2]])


def probabilities(params, X):
    return 1.0 / (1.0 + np.exp(-forward(params, np.asarray(X, np.float64))[2]))


def core_mask(n, ei, ej, prob, threshold, core_fraction):
    """Edges kept by the proposal: confident, both endpoints core nodes
    (confident share of their undirected non-loop edges >= core_fraction)."""
    ei = np.asarray(ei, np.int64)
    ej = np.asarray(ej, np.int64)
    conf = np.asarray(prob) > threshold
    deg = np.bincount(ei, minlength=n) + np.bincount(ej, minlength=n)
    cd = np.bincount(ei, weights=conf, minlength=n) + np.bincount(ej, weights=conf, minlength=n)
    core = cd >= core_fraction * deg
    return conf & core[ei] & core[ej]


def components(n, ei, ej, mask):
    """Components of the masked edges, ids by ascending smallest member."""
    parent = np.arange(n)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for a, b, keep in zip(ei, ej, mask):
        if keep:
            ra, rb = find(int(a)), find(int(b))
            if ra != rb:
                parent[max(ra, rb)] = min(ra, rb)
    roots = np.array([find(v) for v in range(n)])
    _, lab = np.unique(roots, return_inverse=True)
    return lab.astype(np.uint64)
