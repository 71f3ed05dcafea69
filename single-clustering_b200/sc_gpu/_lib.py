"""Loader and ctypes signatures of libsc_gpu.so (include/sc_gpu.h).

The library is the only implementation behind this package: if it is missing
or the GPU is absent the calls fail loudly, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsc_gpu.so")

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
vp = C.c_void_p
vpp = C.POINTER(C.c_void_p)


class ErrorInfo(C.Structure):
    _fields_ = [
        ("code", C.c_int32),
        ("node", C.c_uint64),
        ("n_nodes", C.c_uint64),
        ("edge_from", C.c_uint64),
        ("edge_to", C.c_uint64),
        ("weight", C.c_double),
        ("got", C.c_uint64),
        ("expected_len", C.c_uint64),
        ("degree_sum", C.c_double),
        ("expected", C.c_double),
        ("message", C.c_char * 256),
    ]


class LeidenConfigC(C.Structure):
    _fields_ = [
        ("objective", C.c_int32),
        ("resolution", C.c_double),
        ("has_seed", C.c_int32),
        ("seed", C.c_uint64),
        ("n_iterations", C.c_uint64),
        ("max_levels", C.c_uint64),
        ("tolerance", C.c_double),
        ("refine", C.c_int32),
        ("refine_randomness", C.c_double),
        ("patience", C.c_uint64),
        ("has_max_community_weight", C.c_int32),
        ("max_community_weight", C.c_double),
    ]


class RunStats(C.Structure):
    _fields_ = [
        ("passes", C.c_uint64),
        ("levels", C.c_uint64),
        ("local_move_sweeps", C.c_uint64),
        ("moves", C.c_uint64),
        ("kernel_launches", C.c_uint64),
        ("ms_local_move", C.c_double),
        ("ms_refine", C.c_double),
        ("ms_aggregate", C.c_double),
        ("ms_other", C.c_double),
        ("ms_total", C.c_double),
        ("alg_bytes_local_move", C.c_double),
        ("alg_bytes_refine", C.c_double),
        ("alg_bytes_aggregate", C.c_double),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("lanes8_max_degree", C.c_uint32),
        ("lanes16_max_degree", C.c_uint32),
        ("lanes32_max_degree", C.c_uint32),
        ("small_batch", C.c_uint32),
    ]


class KnnOpts(C.Structure):
    _fields_ = [
        ("sigma", C.c_int32),
        ("sym", C.c_int32),
        ("precision", C.c_int32),
        ("rerank_factor", C.c_int32),
        ("squared_kiddo", C.c_int32),
    ]


class KnnStats(C.Structure):
    _fields_ = [
        ("clusters", C.c_uint64),
        ("tiles_scanned", C.c_uint64),
        ("tiles_full", C.c_uint64),
        ("tiles_pass1", C.c_uint64),
        ("ms_cluster", C.c_double),
        ("ms_pass1", C.c_double),
        ("ms_bounds", C.c_double),
        ("ms_pass2", C.c_double),
    ]


# (name, restype, argtypes) of every symbol include/sc_gpu.h declares
SIGNATURES = [
    ("sc_abi_version", C.c_uint32, []),
    ("sc_ctx_create", C.c_int, [C.c_int32, vpp]),
    ("sc_ctx_destroy", None, [vp]),
    ("sc_last_error_message", C.c_char_p, [vp]),
    ("sc_last_error_info", C.c_int, [vp, C.POINTER(ErrorInfo)]),
    ("sc_last_run_stats", C.c_int, [vp, C.POINTER(RunStats)]),
    ("sc_ctx_synchronize", C.c_int, [vp]),
    ("sc_tuning_default", None, [C.POINTER(Tuning)]),
    ("sc_get_tuning", C.c_int, [vp, C.POINTER(Tuning)]),
    ("sc_set_tuning", C.c_int, [vp, C.POINTER(Tuning)]),
    ("sc_set_wait_limit", C.c_int, [vp, C.c_uint32]),
    ("sc_get_wait_limit", C.c_int, [vp, C.POINTER(C.c_uint32)]),
    ("sc_test_knn_hold_tiles", C.c_int, [vp, C.c_int32]),
    ("sc_set_knn_clusters", C.c_int, [vp, C.c_uint32]),
    ("sc_knn_last_stats", C.c_int, [vp, C.POINTER(KnnStats)]),
    ("sc_knn_autotune", C.c_int, [vp, f32p, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(KnnOpts),
                                  C.POINTER(C.c_uint32), f64p, f64p, C.POINTER(C.c_uint32)]),
    ("sc_autotune", C.c_int, [vp, vp, C.POINTER(LeidenConfigC), C.POINTER(Tuning), f64p, f64p,
                              C.POINTER(C.c_uint32)]),
    ("sc_leiden_config_default", None, [C.POINTER(LeidenConfigC)]),
    ("sc_graph_from_csr", C.c_int, [vp, u64p, C.c_uint64, u32p, C.c_uint64, f32p, C.c_uint64, f64p,
                                     C.c_uint64, vpp]),
    ("sc_graph_from_csr_device", C.c_int, [vp, vp, C.c_uint64, vp, C.c_uint64, vp, C.c_uint64, vp,
                                            C.c_uint64, vpp]),
    ("sc_graph_from_edges", C.c_int, [vp, C.c_uint64, u64p, u64p, f64p, C.c_uint64, f64p, vpp]),
    ("sc_graph_from_csr_matrix", C.c_int, [vp, u64p, C.c_uint64, u64p, f64p, C.c_uint64, f64p, vpp]),
    ("sc_graph_destroy", None, [vp]),
    ("sc_graph_info", C.c_int, [vp, u64p, u64p, u64p, f64p, i32p]),
    ("sc_graph_set_embedding", C.c_int, [vp, vp, f32p, C.c_uint64, C.c_uint64]),
    ("sc_graph_copy_csr", C.c_int, [vp, vp, u64p, u32p, f32p]),
    ("sc_graph_copy_node_data", C.c_int, [vp, vp, f64p, f64p]),
    ("sc_graph_validate_symmetry", C.c_int, [vp, vp]),
    ("sc_aggregate", C.c_int, [vp, vp, u64p, C.c_uint64, vpp]),
    ("sc_modularity", C.c_int, [vp, vp, u64p, C.c_uint64, C.c_double, f64p]),
    ("sc_quality", C.c_int, [vp, vp, u64p, C.c_uint64, C.c_int32, C.c_double, f64p]),
    ("sc_modularity_static", C.c_int, [vp, vp, vp, C.c_uint64, C.c_double, f64p]),
    ("sc_partition_stats", C.c_int, [vp, vp, u64p, C.c_uint64, u64p, u32p, f64p, f64p, f64p, C.c_uint64]),
    ("sc_leiden", C.c_int, [vp, vp, C.POINTER(LeidenConfigC), u64p, u64p]),
    ("sc_leiden_from", C.c_int, [vp, vp, C.POINTER(LeidenConfigC), u64p, C.c_uint64, u64p, u64p]),
    ("sc_leiden_batch", C.c_int, [vp, C.POINTER(vp), C.POINTER(LeidenConfigC), C.c_uint64, u64p, u64p,
                                  u64p]),
    ("sc_leiden_batch_ex", C.c_int, [vp, C.POINTER(vp), C.POINTER(LeidenConfigC), C.c_uint64,
                                     C.POINTER(C.c_int64), u64p, u64p, u64p, C.c_uint32]),
    ("sc_leiden_batch_union", C.c_int, [vp, C.POINTER(vp), C.POINTER(LeidenConfigC), C.c_uint64,
                                        C.POINTER(C.c_int64), u64p, u64p, u64p, C.c_uint64]),
    ("sc_knn_opts_default", None, [C.POINTER(KnnOpts)]),
    ("sc_knn_gaussian", C.c_int, [vp, f32p, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(KnnOpts), u32p,
                                  f32p, u64p, u32p, f32p, C.c_uint64, u64p, vpp]),
    ("sc_knn_search", C.c_int, [vp, f32p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                C.POINTER(KnnOpts), u32p, f32p]),
    ("sc_knn_connectivities", C.c_int, [vp, u32p, f32p, C.c_uint64, C.c_uint64, C.POINTER(KnnOpts), u64p, u32p,
                                        f32p, C.c_uint64, u64p, vpp]),
    ("sc_mlp_param_count", C.c_uint32, []),
    ("sc_mlp_feature_count", C.c_uint32, []),
    ("sc_mlp_create", C.c_int, [vp, C.c_uint64, vpp]),
    ("sc_mlp_destroy", None, [vp]),
    ("sc_mlp_get", C.c_int, [vp, vp, f32p, f32p, i32p]),
    ("sc_mlp_set", C.c_int, [vp, vp, f32p, f32p]),
    ("sc_mlp_features", C.c_int, [vp, vp, vp, C.c_double, u64p, u64p, f32p, u32p, u32p, C.c_uint64, u64p]),
    ("sc_mlp_train", C.c_int, [vp, vp, vp, u64p, C.c_uint64, C.c_double, u64p, u64p, C.c_uint32, C.c_double, f64p,
                               f32p]),
    ("sc_mlp_propose", C.c_int, [vp, vp, vp, C.c_double, u64p, u64p, C.c_double, C.c_double, u64p, u64p, f32p,
                                 C.c_uint64]),
]

_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"{LIB_PATH} is missing: build it with single-clustering_b200/build.py "
                        "(there is no CPU fallback)")
                L = C.CDLL(LIB_PATH)
                for name, res, args in SIGNATURES:
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


_tls = threading.local()


class Context:
    """One sc_ctx (CUDA stream + memory pool + last error) per host thread."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        rc = lib().sc_ctx_create(device, C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"sc_ctx_create(device={device}) failed with status {rc}; "
                               "a CUDA GPU is required")
        self.device = device

    def __del__(self):
        try:
            if self.h:
                lib().sc_ctx_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def error_info(self) -> ErrorInfo:
        info = ErrorInfo()
        lib().sc_last_error_info(self.h, C.byref(info))
        return info

    def run_stats(self) -> dict:
        s = RunStats()
        lib().sc_last_run_stats(self.h, C.byref(s))
        return {name: getattr(s, name) for name, _ in RunStats._fields_}


def context(device: int | None = None) -> Context:
    dev = 0 if device is None else device
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if dev not in ctxs:
        ctxs[dev] = Context(dev)
    return ctxs[dev]
