"""sc_modularity_static: modularity with no device allocation.

Some callers cannot call cudaMalloc — a host framework that already owns the
device's memory through its own pool, a hard device-memory budget, or a code
section where an allocation's implicit synchronisation is not allowed. For
them the library offers sc_modularity_static, which uses only the memory the
caller passes in (graph handle, device labels, host output) and a fixed 1 MiB
scratch array inside the library.

This test calls it through the C ABI with labels the test placed on the device
itself, twice in a row (the scratch keeps the previous call's contents, so the
second call checks that everything it accumulates into is cleared), and
compares each result bit for bit with sc_modularity, the allocating entry
point, as the other modularity parity tests do. The file is named so pytest
collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_labels(labels):
    import torch
    return torch.as_tensor(np.asarray(labels, dtype=np.int64).astype(np.int32), device="cuda:0")


def _static_modularity(g, d_labels, n, gamma):
    from sc_gpu import _lib
    out = C.c_double()
    rc = _lib.lib().sc_modularity_static(g._ctx.h, g._h, C.c_void_p(d_labels.data_ptr()), n, gamma,
                                          C.byref(out))
    return rc, out.value


def _graphs():
    import sc_gpu
    from sc_gpu import synth
    from helpers import karate
    edges, opt = karate()
    k = sc_gpu.CSRNetwork.from_edges(34, edges)
    src, dst, w, truth = synth.planted_partition()
    p = sc_gpu.CSRNetwork.from_edge_arrays(20000, src, dst, w)
    lab = sc_gpu.leiden(p, sc_gpu.LeidenConfig(seed=3)).labels()
    return [(k, opt), (p, truth), (p, lab), (p, np.arange(20000) % 997)]


def test_static_modularity_matches_allocating_entry_point_twice():
    import sc_gpu
    for g, labels in _graphs():
        n = g.node_count()
        d = _device_labels(labels)
        for gamma in (1.0, 0.5):
            want = sc_gpu.modularity(g, labels, gamma)
            for _ in range(2):
                rc, got = _static_modularity(g, d, n, gamma)
                assert rc == 0
                assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (got, want)


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
    err, free, _total = rt.cudaMemGetInfo()
    assert int(err) == 0
    return int(free)


def test_static_modularity_allocates_nothing():
    """The property the entry point exists for: after one warm-up call (which
    loads the kernels and looks up the scratch address), further calls leave the
    device's default pool (where every other entry point of the library takes
    its temporaries) and the device's free memory exactly as they were."""
    import sc_gpu
    from sc_gpu import synth
    src, dst, w, truth = synth.planted_partition()
    g = sc_gpu.CSRNetwork.from_edge_arrays(20000, src, dst, w)
    d = _device_labels(truth)
    rc, first = _static_modularity(g, d, 20000, 1.0)
    assert rc == 0
    used0, free0 = _pool_used(), _device_free()
    for gamma in (1.0, 0.5, 2.0, 1.0, 1.0):
        rc, got = _static_modularity(g, d, 20000, gamma)
        assert rc == 0
    used1, free1 = _pool_used(), _device_free()
    assert used1 == used0, (used0, used1)
    assert free1 == free0, (free0, free1)
    assert got == first


def test_static_modularity_rejects_labels_past_its_limit():
    import sc_gpu
    from sc_gpu import _lib
    g = sc_gpu.CSRNetwork.from_edges(3, [(0, 1, 1.0), (1, 2, 1.0)])
    rc, _ = _static_modularity(g, _device_labels([0, 1, 70000]), 3, 1.0)
    assert rc == 25  # SC_E_UNSUPPORTED
    msg = _lib.lib().sc_last_error_message(g._ctx.h).decode()
    assert "65536" in msg
    # still usable afterwards
    rc, got = _static_modularity(g, _device_labels([0, 0, 1]), 3, 1.0)
    assert rc == 0 and got == sc_gpu.modularity(g, [0, 0, 1], 1.0)
