"""Host logic of multi-GPU sharding, on CPU: the dealing rules; two gloo ranks
that shard a sweep, run their shares with the CPU oracle standing in for the
GPU runner, and all-gather the labels; two gloo ranks that split a kNN search
by query rows (FP64 oracle search standing in for sc_knn_search) and gather
the lists."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sc_gpu import parallel, sweep_plan


def test_chains_and_deal():
    warm = [-1, 0, 1, -1, 3, -1]
    assert parallel.chains(warm) == [[0, 1, 2], [3, 4], [5]]
    assert parallel.deal([5, 1, 4, 2], 2) == [[0, 1], [2, 3]]
    parts = parallel.shard(warm, [1, 1, 1, 1, 1, 1], 2)
    assert sorted(parts[0] + parts[1]) == list(range(6))
    assert parts == [[0, 1, 2], [3, 4, 5]]


def test_sweep_plan_chains_descending_resolutions():
    cfgs, warm, keys = sweep_plan([0.5, 2.0, 1.0], [1, 2])
    assert [k[0] for k in keys[:3]] == [2.0, 1.0, 0.5]
    assert warm == [-1, 0, 1, -1, 3, 4]
    assert all(c.seed == k[1] and c.objective.resolution == k[0] for c, k in zip(cfgs, keys))
    _, warm_plain, _ = sweep_plan([0.5, 2.0], [1], warm_start=False)
    assert warm_plain == [-1, -1]
    # split chains: pieces [0..2] [3..4] [5..7] of 8 resolutions (bounds round(i*8/3));
    # piece heads warm from the seed's first (finest) instance
    _, warm_split, keys = sweep_plan([float(x) for x in range(1, 9)], [1, 2], split=3)
    assert warm_split[:8] == [-1, 0, 1, 0, 3, 0, 5, 6]
    assert warm_split[8:] == [-1, 8, 9, 8, 11, 8, 13, 14]
    assert [k[0] for k in keys[:8]] == [8.0, 7.0, 6.0, 5.0, 4.0, 3.0, 2.0, 1.0]
    assert parallel.chains(warm_split) == [list(range(8)), list(range(8, 16))]
    # warm-started instances run one pass by default (their start replaces the
    # plain run's first pass); chain heads keep the base config's passes
    assert [c.n_iterations for c in cfgs] == [2, 1, 1, 2, 1, 1]
    cfgs2, _, _ = sweep_plan([0.5, 2.0, 1.0], [1], warm_passes=None)
    assert [c.n_iterations for c in cfgs2] == [2, 2, 2]
    cfgs3, _, _ = sweep_plan([0.5, 2.0], [1], warm_start=False)
    assert [c.n_iterations for c in cfgs3] == [2, 2]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle as O
    from helpers import sbm
    edges, _ = sbm(20, 4, 0.4, 0.02, 7)
    g = O.Graph.from_edges(80, edges)
    cfgs, warm, keys = sweep_plan([0.5, 1.0, 2.0], [1, 2, 3])

    def run_local(ids, local_warm):
        out = []
        for k, gid in enumerate(ids):
            c = cfgs[gid]
            ini = out[local_warm[k]][0] if local_warm[k] >= 0 else None
            lab, ncl = g.leiden(seed=c.seed, resolution=c.objective.resolution, initial=ini)
            out.append((lab, ncl))
        return out

    res = parallel.run_sharded(run_local, len(cfgs), warm, [1.0] * len(cfgs), rank, world)
    q.put((rank, [(int(r[1]), r[0].tolist()) for r in res]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_same_sweep():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1]
    assert len(out[0]) == 9 and all(k >= 1 for k, _ in out[0])


def test_row_blocks_cover_rows_once():
    for n, world in ((10, 3), (7, 8), (0, 2), (1_000_003, 8)):
        blocks = parallel.row_blocks(n, world)
        assert len(blocks) == world and blocks[0][0] == 0 and blocks[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
        sizes = [e - b for b, e in blocks]
        assert max(sizes) - min(sizes) <= 1


def _knn_rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import knn_oracle as K
    rng = np.random.default_rng(3)
    X = rng.normal(size=(301, 5)).astype(np.float32)
    full_idx, full_d = K.knn_exact(X, 6)

    def search(b, e):
        return full_idx[b:e].astype(np.uint32), (full_d[b:e] ** 2).astype(np.float32)

    idx, d2 = parallel.knn_sharded(search, len(X), rank, world)
    q.put((rank, idx.tolist(), d2.tolist(), full_idx.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_knn_lists():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_knn_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {r: (i, d, f) for r, i, d, f in (q.get(timeout=120) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert out[0][0] == out[0][2]
