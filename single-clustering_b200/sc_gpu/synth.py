"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is used anywhere: every workload is drawn from numpy's
PCG64 with a recorded seed, so the CPU oracle and the GPU path see identical
bytes.
"""
from __future__ import annotations

import numpy as np


def planted_partition(n: int = 20_000, blocks: int = 40, intra: int = 12, inter: int = 3,
                      seed: int = 1, w_lo: float = 0.5, w_hi: float = 1.5):
    """Planted-partition edge list: each node draws `intra` partners inside its
    block and `inter` partners outside it, uniformly; weights f32 U[w_lo, w_hi].

    Returns (src u64, dst u64, w f64 holding f32 values, truth labels). Duplicate
    pairs are left in: `from_edges` merges them by summing (csr_network.rs:104-109).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    per = n // blocks
    node = np.arange(n, dtype=np.int64)
    block = np.minimum(node // per, blocks - 1)
    base = block * per
    size = np.where(block == blocks - 1, n - base, per)
    src_a = np.repeat(node, intra)
    off = rng.integers(1, np.repeat(size, intra), dtype=np.int64)
    dst_a = base[src_a] + ((src_a - base[src_a]) + off) % size[src_a]
    src_b = np.repeat(node, inter)
    outside = n - size[src_b]
    r = rng.integers(0, outside, dtype=np.int64)
    dst_b = np.where(r < base[src_b], r, r + size[src_b])
    src = np.concatenate([src_a, src_b]).astype(np.uint64)
    dst = np.concatenate([dst_a, dst_b]).astype(np.uint64)
    w = rng.uniform(w_lo, w_hi, size=src.shape[0]).astype(np.float32).astype(np.float64)
    return src, dst, w, block.astype(np.uint64)


def many_planted_graphs(count: int = 512, seed: int = 21, n_range=(100, 50_000), blocks_range=(5, 200),
                        degree_range=(10.0, 30.0), intra_share: float = 0.8):
    """Many independent planted-partition graphs: node counts log-uniform in
    n_range, block counts uniform in blocks_range (at most n/5), mean degree
    uniform in degree_range with intra_share of each node's draws inside its
    block, f32 weights U[0.5, 1.5]. Yields (n, src, dst, w, truth) per graph."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]), count)).astype(np.int64)
    bs = rng.integers(blocks_range[0], blocks_range[1] + 1, count)
    ds = rng.uniform(degree_range[0], degree_range[1], count)
    for i in range(count):
        n = int(ns[i])
        blocks = int(max(1, min(bs[i], n // 5)))
        draws = ds[i] / 2.0  # each draw adds one entry to both endpoints' rows
        intra = max(1, int(round(intra_share * draws)))
        inter = max(0, int(round(draws)) - intra)
        src, dst, w, truth = planted_partition(n, blocks, intra, inter, seed * 100_003 + i)
        yield n, src, dst, w, truth


def gaussian_mixture(n: int, d: int, components: int, seed: int, sigma=(1.0, 1.0),
                     centre_scale: float = 2.0):
    """Isotropic Gaussian mixture, f32 row-major [n, d]: centres ~ N(0, centre_scale^2 I),
    per-component sigma ~ U[sigma], mixture weights ~ Dirichlet(1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.normal(0.0, centre_scale, size=(components, d))
    sig = rng.uniform(sigma[0], sigma[1], size=components)
    pi = rng.dirichlet(np.ones(components))
    comp = rng.choice(components, size=n, p=pi)
    x = np.empty((n, d), dtype=np.float32)
    chunk = 1 << 20
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        c = comp[s:e]
        x[s:e] = (centres[c] + rng.standard_normal((e - s, d)) * sig[c, None]).astype(np.float32)
    return x, comp.astype(np.uint64)


def knn_like_graph(n: int, k: int = 10, blocks: int = 100, seed: int = 7):
    """A symmetrised kNN-shaped CSR without a full kNN search: points on a 2-D
    jittered lattice per block, each linked to k lattice neighbours; Gaussian
    weights of the lattice distance. Returns (ptrs u64, nbrs u32, w f32)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    side = int(np.ceil(np.sqrt(n)))
    idx = np.arange(n, dtype=np.int64)
    gx, gy = idx % side, idx // side
    offs = [(1, 0), (0, 1), (1, 1), (1, -1), (2, 0), (0, 2), (2, 1), (1, 2), (2, -1), (1, -2)]
    offs = offs[: max(1, k // 2 + k % 2)]
    src_l, dst_l = [], []
    for dx, dy in offs:
        nx, ny = gx + dx, gy + dy
        ok = (nx >= 0) & (nx < side) & (ny >= 0)
        j = ny * side + nx
        ok &= j < n
        src_l.append(idx[ok])
        dst_l.append(j[ok])
    src = np.concatenate(src_l)
    dst = np.concatenate(dst_l)
    # random long-range rewiring keeps it from being a pure lattice
    rew = rng.random(src.shape[0]) < 0.02
    dst[rew] = rng.integers(0, n, size=int(rew.sum()))
    keep = src != dst
    src, dst = src[keep], dst[keep]
    lo, hi = np.minimum(src, dst), np.maximum(src, dst)
    key = np.unique(lo * n + hi)
    lo, hi = key // n, key % n
    d2 = ((gx[lo] - gx[hi]) ** 2 + (gy[lo] - gy[hi]) ** 2).astype(np.float64)
    w = np.exp(-d2 / 4.0) * rng.uniform(0.6, 1.0, size=lo.shape[0])
    rows = np.concatenate([lo, hi])
    cols = np.concatenate([hi, lo])
    ww = np.concatenate([w, w]).astype(np.float32)
    order = np.lexsort((cols, rows))
    rows, cols, ww = rows[order], cols[order], ww[order]
    ptrs = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(rows, minlength=n), out=ptrs[1:])
    return ptrs, cols.astype(np.uint32), ww


def knn_graph_exact_torch(X, groups, k: int, device, chunk: int = 4096, margin: int = 8):
    """Exact kNN graph of the points X built with torch alone (no call into this
    library), for benchmark inputs that must not depend on the code under test:
    k nearest points by FP64 distance (ties by lower index, the point itself
    first), Gaussian weights with sigma = the k-th neighbour's distance
    (w = sqrt(2 s_i s_j / (s_i^2 + s_j^2)) exp(-d^2 / (s_i^2 + s_j^2)), kept if
    > 1e-14), union symmetrisation, f32 weights. Returns (ptrs u64, nbrs u32,
    w f32, index (n, k+1) int64, dist (n, k+1) float64).

    `groups` (one id per point, e.g. the mixture component) only organises the
    search; the result is exact whatever the grouping. Each query first searches
    its own group; then group h is searched by exactly the queries whose lower
    bound on the distance to any member of h is at most their current k-th
    distance. The bound is the larger of a ball bound (distance to h's centre
    minus h's radius) and a slab bound: with u the unit vector from the query's
    group centre to h's, every member x of h projects into [lo, hi] on u, and
    |q - x| >= the distance from <q, u> to that interval. Candidates come from
    FP32 scores |c|^2 - 2 q.c (TF32 off) with `margin` spares, then exact FP64
    differences rank them."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    X = np.ascontiguousarray(X, dtype=np.float32)
    groups = np.asarray(groups)
    n, d = X.shape
    order = np.argsort(groups, kind="stable")
    gs = groups[order]
    bounds = np.flatnonzero(np.r_[True, gs[1:] != gs[:-1], True])
    starts, ends = bounds[:-1].tolist(), bounds[1:].tolist()
    G = len(starts)
    x32 = torch.from_numpy(X[order]).to(device)
    x64 = x32.to(torch.float64)
    orig = torch.from_numpy(order.astype(np.int64)).to(device)
    nrm32 = (x32 * x32).sum(1)
    gid = torch.empty(n, dtype=torch.int64, device=device)
    for g, (a, b) in enumerate(zip(starts, ends)):
        gid[a:b] = g
    cen = torch.stack([x64[a:b].mean(0) for a, b in zip(starts, ends)])
    rad = torch.stack([((x64[a:b] - cen[g]) ** 2).sum(1).max().sqrt() for g, (a, b) in enumerate(zip(starts, ends))])
    # unit directions between group centres (zero when two centres coincide)
    diff = cen[None, :, :] - cen[:, None, :]
    ln = diff.norm(dim=2, keepdim=True)
    U = torch.where(ln > 0, diff / torch.where(ln > 0, ln, torch.ones_like(ln)), torch.zeros_like(diff))  # U[a, h]
    lo = torch.empty((G, G), dtype=torch.float64, device=device)
    hi = torch.empty((G, G), dtype=torch.float64, device=device)
    for h, (a, b) in enumerate(zip(starts, ends)):
        pr = x64[a:b] @ U[:, h, :].T  # (|h|, G): member projections on every u_{g,h}
        lo[:, h] = pr.min(0).values
        hi[:, h] = pr.max(0).values
    kk = k + 1 + margin
    best_i = torch.empty((n, k + 1), dtype=torch.int64, device=device)  # sorted positions
    best_d = torch.empty((n, k + 1), dtype=torch.float64, device=device)

    def candidates(qpos, a, b):
        """FP32 top-kk positions in [a, b) for the queries at sorted positions qpos."""
        out = []
        for s in range(0, len(qpos), chunk):
            qp = qpos[s:s + chunk]
            sc = torch.addmm(nrm32[None, a:b], x32[qp], x32[a:b].T, beta=1.0, alpha=-2.0)
            _, j = torch.topk(sc, min(kk, b - a), dim=1, largest=False)
            out.append(j + a)
        return torch.cat(out)

    def rank(qpos, cand):
        """Exact FP64 (distance, self first, original index) order of the candidate
        positions (-1: an empty slot, ordered last); returns the first k+1 as
        (positions, d2), empty slots as (-1, +inf)."""
        valid = cand >= 0
        cc = cand.clamp(min=0)
        dd = ((x64[cc] - x64[qpos][:, None, :]) ** 2).sum(-1)
        dd = torch.where(valid, dd, torch.full_like(dd, float("inf")))
        oi = torch.where(valid, orig[cc], torch.full_like(cc, n))
        o = torch.argsort(oi, dim=1, stable=True)
        cand, dd, oi = torch.gather(cand, 1, o), torch.gather(dd, 1, o), torch.gather(oi, 1, o)
        o = torch.argsort((oi != orig[qpos][:, None]).to(torch.int8), dim=1, stable=True)
        cand, dd = torch.gather(cand, 1, o), torch.gather(dd, 1, o)
        o = torch.argsort(dd, dim=1, stable=True)
        cand, dd = torch.gather(cand, 1, o)[:, : k + 1], torch.gather(dd, 1, o)[:, : k + 1]
        if cand.shape[1] < k + 1:
            pad = k + 1 - cand.shape[1]
            cand = torch.cat([cand, torch.full((len(qpos), pad), -1, dtype=torch.int64, device=device)], 1)
            dd = torch.cat([dd, torch.full((len(qpos), pad), float("inf"), dtype=torch.float64, device=device)], 1)
        cand = torch.where(torch.isfinite(dd), cand, torch.full_like(cand, -1))
        return cand, dd

    # 1) every query against its own group
    for g, (a, b) in enumerate(zip(starts, ends)):
        qpos = torch.arange(a, b, device=device)
        c, dd = rank(qpos, candidates(qpos, a, b))
        best_i[a:b], best_d[a:b] = c, dd
    # 2) every other group h, searched by the queries whose bound does not exclude it
    kth = best_d[:, k].sqrt()
    for h, (a, b) in enumerate(zip(starts, ends)):
        ga = gid  # the query's own group
        pq = (x64 * U[ga, h, :]).sum(1)
        slab = torch.clamp(torch.maximum(lo[ga, h] - pq, pq - hi[ga, h]), min=0.0)
        ball = torch.clamp((x64 - cen[h]).norm(dim=1) - rad[h], min=0.0)
        lb = torch.maximum(slab, ball) * (1.0 - 1e-9)
        need = (lb <= kth) & (ga != h)
        qpos = torch.nonzero(need).flatten()
        if len(qpos) == 0:
            continue
        # the current best (from groups searched before, never h) and h's candidates
        cand = torch.cat([best_i[qpos], candidates(qpos, a, b)], 1)
        best_i[qpos], best_d[qpos] = rank(qpos, cand)
    out_i = torch.empty((n, k + 1), dtype=torch.int64, device=device)
    out_d = torch.empty((n, k + 1), dtype=torch.float64, device=device)
    out_i[orig] = torch.where(best_i >= 0, orig[best_i.clamp(min=0)], torch.full_like(best_i, -1))
    out_d[orig] = best_d.sqrt()
    sig = out_d[:, k]
    rows = torch.arange(n, device=device).repeat_interleave(k)
    cols = out_i[:, 1:].reshape(-1)
    dd = out_d[:, 1:].reshape(-1)
    si, sj = sig[rows], sig[cols]
    den = si * si + sj * sj
    w = torch.sqrt(2 * si * sj / den) * torch.exp(-dd * dd / den)
    keep = (rows != cols) & (w > 1e-14)
    rows, cols, w = rows[keep], cols[keep], w[keep]
    lo_, hi_ = torch.minimum(rows, cols), torch.maximum(rows, cols)
    key, o = torch.sort(lo_ * n + hi_, stable=True)
    w = w[o]
    first = torch.ones_like(key, dtype=torch.bool)
    first[1:] = key[1:] != key[:-1]
    key, w = key[first], w[first]
    lo_, hi_ = key // n, key % n
    r = torch.cat([lo_, hi_])
    c = torch.cat([hi_, lo_])
    ww = torch.cat([w, w]).float()
    _, o = torch.sort(r * n + c)
    r, c, ww = r[o], c[o], ww[o]
    ptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    ptr[1:] = torch.cumsum(torch.bincount(r, minlength=n), 0)
    res = (ptr.cpu().numpy().astype(np.uint64), c.to(torch.int32).cpu().numpy().view(np.uint32).copy(),
           ww.cpu().numpy(), out_i.cpu().numpy(), out_d.cpu().numpy())
    del x32, x64, out_i, out_d, best_i, best_d
    if str(device).startswith("cuda"):
        torch.cuda.empty_cache()
    return res

