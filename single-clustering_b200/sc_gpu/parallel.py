"""Multi-GPU sharding of independent Leiden instances and of the kNN search.

A single graph does not shard (every move reads global community statistics),
so one graph runs as replicas. A resolution x seed sweep or a set of many
graphs is made of independent units: whole warm-start chains (or single
instances) are dealt to ranks by estimated cost, each rank runs its share on
its own GPU with `leiden_batch`, and the labels are gathered with one
all-gather of Python objects over the process group (NCCL over NVLink between
GPUs, gloo on CPU). No collective runs inside a Leiden run.

The kNN search shards by query rows: every rank holds all points, searches
its contiguous block of rows (`knn_search`), and a tensor all-gather of the
k+1 lists (ids and squared distances) lets every rank build the
connectivities (`knn_connectivities`).
"""
from __future__ import annotations

from typing import Callable, Sequence


def chains(warm_from: Sequence[int]) -> list:
    """Instance ids grouped into warm-start chains (a chain never splits)."""
    owner = {}
    out = []
    for i, j in enumerate(warm_from):
        if j is None or j < 0:
            owner[i] = len(out)
            out.append([i])
        else:
            owner[i] = owner[j]
            out[owner[j]].append(i)
    return out


def deal(costs: Sequence[float], world: int) -> list:
    """Longest-processing-time-first assignment of units to `world` ranks:
    the costliest unit goes to the least loaded rank, ties to the lower rank."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for u in sorted(range(len(costs)), key=lambda u: (-costs[u], u)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(u)
        load[r] += costs[u]
    return [sorted(p) for p in parts]


def shard(warm_from: Sequence[int], instance_cost: Sequence[float], world: int) -> list:
    """Instance ids per rank: chains dealt whole by their summed cost."""
    ch = chains(warm_from)
    parts = deal([sum(instance_cost[i] for i in c) for c in ch], world)
    return [sorted(i for u in p for i in ch[u]) for p in parts]


def run_sharded(run_local: Callable, n_instances: int, warm_from: Sequence[int],
                instance_cost: Sequence[float], rank: int, world: int, group=None) -> list:
    """Runs this rank's instances with run_local(ids, local_warm_from) -> list of
    results (in ids order) and gathers every rank's results: returns the results
    of all n_instances in instance order on every rank."""
    mine = shard(warm_from, instance_cost, world)[rank]
    pos = {g: k for k, g in enumerate(mine)}
    local_warm = [pos[warm_from[g]] if warm_from[g] >= 0 else -1 for g in mine]
    local = run_local(mine, local_warm)
    if world == 1:
        gathered = [(mine, local)]
    else:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, (mine, local), group=group)
    out = [None] * n_instances
    for ids, res in gathered:
        for g, r in zip(ids, res):
            out[g] = r
    return out


def row_blocks(n: int, world: int) -> list:
    """Contiguous query-row blocks [begin, end) per rank, sizes differing by at most one."""
    base, extra = divmod(n, world)
    out, b = [], 0
    for r in range(world):
        e = b + base + (1 if r < extra else 0)
        out.append((b, e))
        b = e
    return out


def knn_sharded(search: Callable, n: int, rank: int, world: int, group=None):
    """search(begin, end) -> (index (end-begin, k+1), squared distances) for this
    rank's rows; returns the (n, k+1) lists of all rows on every rank."""
    import numpy as np
    b, e = row_blocks(n, world)[rank]
    idx, d2 = search(b, e)
    if world == 1:
        return idx, d2
    import torch
    import torch.distributed as dist
    # one tensor all-gather per array (rows padded to the largest block): the
    # ids travel as int32 bit patterns, on the GPU under NCCL, on the host under
    # gloo; nothing is pickled
    blocks = row_blocks(n, world)
    rows = max(hi - lo for lo, hi in blocks)
    kk = idx.shape[1]
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    out = []
    for a, dt in ((np.ascontiguousarray(idx, np.uint32).view(np.int32), torch.int32),
                  (np.ascontiguousarray(d2, np.float32), torch.float32)):
        mine = torch.zeros((rows, kk), dtype=dt, device=dev)
        mine[:e - b] = torch.from_numpy(a).to(dev)
        parts = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine, group=group)
        out.append(np.concatenate([parts[r][:hi - lo].cpu().numpy() for r, (lo, hi) in enumerate(blocks)]))
    return out[0].view(np.uint32), out[1]
