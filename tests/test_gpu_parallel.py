"""The multi-GPU split run by two processes (`gloo` ranks) on the GPU.

This pool gives one GPU per run, so both ranks share it. Their kernels never wait on
each other: each rank runs its own share, and the collectives are host-side `gloo`
operations. Checked:

* `parallel.run_sharded` with the library's `leiden_batch` as the runner: the labels
  of a warm-started resolution x seed sweep equal those of one process running every
  instance (a fixed seed is bit-reproducible);
* `parallel.knn_sharded` with `knn_search` as the search: the gathered lists and the
  connectivities built from them equal the single build's bits.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_NODES, N_POINTS = 4000, 6000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plan():
    import sc_gpu
    return sc_gpu.sweep_plan([0.3, 0.6, 1.0, 1.7, 3.0], [1, 2, 3], sc_gpu.Rb, True, None, 2, 1)


def _graph():
    import sc_gpu
    from sc_gpu import synth
    src, dst, w, _ = synth.planted_partition(N_NODES, 20, 8, 3, 5)
    return sc_gpu.CSRNetwork.from_edge_arrays(N_NODES, src, dst, w)


def _points():
    from sc_gpu import synth
    return synth.gaussian_mixture(N_POINTS, 12, 6, seed=3, sigma=(0.7, 1.5))[0]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    import sc_gpu
    from sc_gpu import parallel
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _graph()
        configs, warm, _ = _plan()

        def run_local(ids, local_warm):
            if not ids:
                return []
            res = sc_gpu.leiden_batch([g] * len(ids), [configs[i] for i in ids], local_warm, 4)
            return [r.labels() for r in res]

        labels = parallel.run_sharded(run_local, len(configs), warm, [1.0] * len(configs), rank, world)
        X = _points()
        idx, d2 = parallel.knn_sharded(lambda b, e: sc_gpu.knn_search(X, 10, b, e), len(X), rank, world)
        r = sc_gpu.knn_connectivities(idx, d2, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION)
        q.put((rank, [np.asarray(x).tolist() for x in labels], idx.tolist(),
               r.conn_ptrs.tolist(), r.conn_nbrs.tolist(), r.conn_w.view(np.uint32).tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_the_gpu_match_one_process():
    import multiprocessing as mp
    import sc_gpu
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, *rest = q.get(timeout=300)
        out[rank] = rest
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # both ranks end with the same gathered results
    assert out[0] == out[1]
    labels, idx, ptrs, nbrs, wbits = out[0]
    # ... and they are the single process's
    g = _graph()
    configs, warm, _ = _plan()
    single = sc_gpu.leiden_batch([g] * len(configs), configs, warm, 4)
    for got, want in zip(labels, single):
        assert np.array_equal(np.asarray(got, np.uint64), want.labels())
    full = sc_gpu.knn_gaussian(_points(), 10, sigma=sc_gpu.SIGMA_KTH, sym=sc_gpu.SYM_UNION)
    assert np.array_equal(np.asarray(idx, np.uint32), full.index)
    assert np.array_equal(np.asarray(ptrs, np.uint64), full.conn_ptrs)
    assert np.array_equal(np.asarray(nbrs, np.uint32), full.conn_nbrs)
    assert np.array_equal(np.asarray(wbits, np.uint32), full.conn_w.view(np.uint32))
