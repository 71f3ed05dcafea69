"""Device memory of destroyed graphs goes back to the device's pool.

Graph arrays come from the stream-ordered pool; a graph dropped by its user
must return them there, or every graph a long-lived process builds stays
allocated (read through the pool's own used-memory counter).
"""
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pool_used():
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert int(err) == 0
    rt.cudaDeviceSynchronize()
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert int(err) == 0
    return int(v)


def _device_free():
    from cuda.bindings import runtime as rt
    rt.cudaDeviceSynchronize()
    err, free, total = rt.cudaMemGetInfo()
    assert int(err) == 0
    return int(free)


def test_destroyed_graphs_return_their_memory():
    import sc_gpu
    rng = np.random.default_rng(3)
    n, k = 200_000, 8
    src = np.repeat(np.arange(n, dtype=np.uint64), k)
    dst = rng.integers(0, n, n * k).astype(np.uint64)
    w = rng.uniform(0.5, 1.5, n * k).astype(np.float32)
    g0 = sc_gpu.CSRNetwork.from_edge_arrays(n, src, dst, w)
    ptr, nbr, ww = g0.to_csr_parts()
    graph_bytes = ptr.nbytes + 3 * nbr.nbytes + 3 * n * 8  # ptr, nbr, w, row ids, three per-node arrays

    def cycle():
        g = sc_gpu.CSRNetwork.from_csr_parts(ptr, nbr, ww)
        labels = sc_gpu.leiden(g).labels()
        sc_gpu.leiden(g.aggregate(labels))  # a pooled aggregate handed to the user, then dropped
        del g
        gc.collect()

    cycle()  # the first cycle settles the run's temporaries in the pool
    before, free_before = _pool_used(), _device_free()
    for _ in range(3):
        cycle()
    after, free_after = _pool_used(), _device_free()
    # three leaked graphs would hold three times graph_bytes
    assert after - before < graph_bytes, (before, after, graph_bytes)
    assert free_before - free_after < graph_bytes, (free_before, free_after, graph_bytes)
