"""FP64 exact kNN + Gaussian connectivities — TEST INFRASTRUCTURE ONLY.

Restates the arithmetic of single-clustering's neighborhood module
(src/neighborhood/mod.rs) on top of an exact FP64 brute-force search. The
reference's own search is third-party code absent here: kiddo 5.2.2 (exact
kd-tree, squared Euclidean distances, :76-89, :233-314) and hnsw_rs 0.3.2
(approximate HNSW, Euclidean distances, :399-448). The reference has no tests
for this module, so parity is anchored on the exact search and on the
formulas below (parity of the search itself is unpinned).

  sigma_i   median of the positive distances among the k+1 (:480-499), or
            sqrt of the median squared distance on the kd-tree path
            (:105-124); 1 if none. ("kth": the k-th neighbour's distance.)
  w_ij      sqrt(2 s_i s_j / (s_i^2 + s_j^2)) * exp(-d_ij^2 / (s_i^2 + s_j^2))
            (:139-163, :513-538), kept if > 1e-14
  emission  lower_id: from row i for each listed j >= i, both directions
            (the reference); union: every listed pair, both directions, once.
"""
from __future__ import annotations

import numpy as np


def knn_exact(X: np.ndarray, k: int, block: int = 2048):
    """Exact k+1 nearest neighbours (self included) in FP64: (idx, dist).

    Rows are ordered by (distance, self first, index)."""
    X64 = np.asarray(X, dtype=np.float64)
    n = X64.shape[0]
    nrm = (X64 * X64).sum(1)
    idx = np.empty((n, k + 1), np.int64)
    dist = np.empty((n, k + 1), np.float64)
    for s in range(0, n, block):
        e = min(n, s + block)
        d2 = nrm[s:e, None] + nrm[None, :] - 2.0 * (X64[s:e] @ X64.T)
        np.maximum(d2, 0.0, out=d2)
        part = np.argpartition(d2, k + 1 if k + 1 < n else n - 1, axis=1)[:, : k + 1] if k + 1 < n else \
            np.tile(np.arange(n), (e - s, 1))
        for r in range(e - s):
            q = s + r
            cand = part[r]
            # exact distances by differences, then (distance, self first, index)
            dd = ((X64[cand] - X64[q]) ** 2).sum(1)
            order = np.lexsort((cand, cand != q, dd))
            idx[q] = cand[order][: k + 1]
            dist[q] = np.sqrt(dd[order][: k + 1])
    return idx, dist


def exact_dist_matrix_rows(X, rows, cols):
    X64 = np.asarray(X, dtype=np.float64)
    return np.sqrt(((X64[rows] - X64[cols]) ** 2).sum(-1))


def sigmas(dist: np.ndarray, kth: bool = False) -> np.ndarray:
    """Per-row sigma over the neighbours actually returned (finite entries; a
    search over fewer than k + 1 points returns fewer)."""
    out = np.ones(dist.shape[0])
    for i, row in enumerate(dist):
        row = row[np.isfinite(row)]
        if kth:
            out[i] = row[-1] if len(row) else 1.0
            continue
        pos = np.sort(row[row > 0])
        if len(pos):
            out[i] = pos[len(pos) // 2]
    return out


def connectivities(idx: np.ndarray, dist: np.ndarray, sigma: np.ndarray, union: bool = False):
    """COO (rows, cols, w) of the Gaussian connectivities, sorted by (row, col)."""
    n, k1 = idx.shape
    pairs = {}
    for i in range(n):
        for t in range(1, k1):
            j = int(idx[i, t])
            if j >= n:  # an empty slot (fewer points than k + 1)
                continue
            if union:
                if j == i:
                    continue
            elif not i <= j:
                continue
            si, sj = sigma[i], sigma[j]
            den = si * si + sj * sj
            if den <= 0:
                continue
            w = np.sqrt(2 * si * sj / den) * np.exp(-dist[i, t] ** 2 / den)
            if not w > 1e-14:
                continue
            pairs[(i, j)] = w
            if i != j:
                pairs[(j, i)] = w
    keys = sorted(pairs)
    rows = np.array([a for a, _ in keys], np.int64)
    cols = np.array([b for _, b in keys], np.int64)
    w = np.array([pairs[x] for x in keys], np.float64)
    return rows, cols, w


def recall(found_idx: np.ndarray, true_idx: np.ndarray) -> float:
    hit = 0
    for a, b in zip(found_idx, true_idx):
        hit += len(set(a.tolist()) & set(b.tolist()))
    return hit / true_idx.size
