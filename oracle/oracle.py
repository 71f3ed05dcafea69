"""ctypes binding of the CPU oracle (liboracle_sc.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py as the checker. The product path never
imports this module.

The oracle restates single-clustering v0.7.0's Leiden path in C++ (see
sc_oracle.cpp for the file:line each function follows).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_sc.so")

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_vp = C.c_void_p

RB, CPM = 0, 1


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


class LeidenConfig(C.Structure):
    """Mirror of ``sc_leiden_config`` (include/sc_gpu.h)."""

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

    @classmethod
    def make(cls, objective=RB, resolution=1.0, seed=42, n_iterations=2, max_levels=64,
             tolerance=1e-9, refine=True, refine_randomness=0.01, patience=2,
             max_community_weight=None):
        c = cls()
        c.objective = objective
        c.resolution = resolution
        c.has_seed = 0 if seed is None else 1
        c.seed = 0 if seed is None else seed
        c.n_iterations = n_iterations
        c.max_levels = max_levels
        c.tolerance = tolerance
        c.refine = 1 if refine else 0
        c.refine_randomness = refine_randomness
        c.patience = patience
        c.has_max_community_weight = 0 if max_community_weight is None else 1
        c.max_community_weight = 0.0 if max_community_weight is None else max_community_weight
        return c


class OracleError(Exception):
    def __init__(self, code: int, info: ErrorInfo):
        self.code = code
        self.info = info
        super().__init__(f"oracle error {code}: {info.message.decode(errors='replace')}")


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_last_error.restype = C.POINTER(ErrorInfo)
        L.orc_graph_from_edges.argtypes = [C.c_uint64, _u64p, _u64p, _f64p, C.c_uint64, _f64p,
                                           C.POINTER(_vp)]
        L.orc_graph_from_csr.argtypes = [_u64p, C.c_uint64, _u32p, C.c_uint64, _f32p, C.c_uint64,
                                         _f64p, C.c_uint64, C.POINTER(_vp)]
        L.orc_graph_from_csr_matrix.argtypes = [_u64p, C.c_uint64, _u64p, _f64p, C.c_uint64,
                                                _f64p, C.POINTER(_vp)]
        L.orc_graph_free.argtypes = [_vp]
        L.orc_graph_info.argtypes = [_vp, _u64p, _u64p, _u64p, _f64p, C.POINTER(C.c_int32)]
        L.orc_graph_arrays.argtypes = [_vp, _u64p, _u32p, _f32p, _f64p, _f64p]
        L.orc_validate_symmetry.argtypes = [_vp]
        L.orc_aggregate.argtypes = [_vp, _u64p, C.c_uint64, C.POINTER(_vp)]
        L.orc_partition_stats.argtypes = [_vp, _u64p, C.c_uint64, _u64p, _u32p, _f64p, _f64p,
                                          _f64p, C.c_uint64]
        L.orc_quality.argtypes = [_vp, _u64p, C.c_uint64, C.c_int32, C.c_double, _f64p]
        L.orc_modularity.argtypes = [_vp, _u64p, C.c_uint64, C.c_double, _f64p]
        L.orc_local_move.argtypes = [_vp, _u64p, C.c_uint64, C.c_int32, C.c_double, C.c_uint64,
                                     C.c_int32, C.c_double, _f64p]
        L.orc_refine.argtypes = [_vp, _u32p, C.c_uint64, C.c_int32, C.c_double, C.c_uint64,
                                 C.c_int32, C.c_double, C.c_double, _u64p]
        L.orc_leiden.argtypes = [_vp, C.POINTER(LeidenConfig), _u64p, _u64p, _u64p]
        _lib = L
    return _lib


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _check(rc):
    if rc != 0:
        raise OracleError(rc, lib().orc_last_error().contents)


class Graph:
    """A CSRNetwork built by the oracle (csr_network.rs:62-69)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    def __del__(self):
        try:
            if self._h:
                lib().orc_graph_free(self._h)
                self._h = None
        except Exception:
            pass

    @classmethod
    def from_edges(cls, n_nodes, edges=None, *, src=None, dst=None, w=None, node_weights=None):
        if edges is not None:
            edges = list(edges)
            src = np.array([e[0] for e in edges], dtype=np.uint64)
            dst = np.array([e[1] for e in edges], dtype=np.uint64)
            w = np.array([e[2] for e in edges], dtype=np.float64)
        src = np.ascontiguousarray(src, dtype=np.uint64)
        dst = np.ascontiguousarray(dst, dtype=np.uint64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        nw = None if node_weights is None else np.ascontiguousarray(node_weights, np.float64)
        h = C.c_void_p()
        _check(lib().orc_graph_from_edges(n_nodes, _p(src, _u64p), _p(dst, _u64p), _p(w, _f64p),
                                          len(src), _p(nw, _f64p), C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr_parts(cls, ptrs, nbrs, w, node_weights=None):
        ptrs = np.ascontiguousarray(ptrs, dtype=np.uint64)
        nbrs = np.ascontiguousarray(nbrs, dtype=np.uint32)
        w = np.ascontiguousarray(w, dtype=np.float32)
        nw = None if node_weights is None else np.ascontiguousarray(node_weights, np.float64)
        h = C.c_void_p()
        _check(lib().orc_graph_from_csr(_p(ptrs, _u64p), len(ptrs), _p(nbrs, _u32p), len(nbrs),
                                        _p(w, _f32p), len(w), _p(nw, _f64p),
                                        0 if nw is None else len(nw), C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr_matrix(cls, indptr, indices, data, node_weights=None):
        indptr = np.ascontiguousarray(indptr, dtype=np.uint64)
        indices = np.ascontiguousarray(indices, dtype=np.uint64)
        data = np.ascontiguousarray(data, dtype=np.float64)
        nw = None if node_weights is None else np.ascontiguousarray(node_weights, np.float64)
        h = C.c_void_p()
        _check(lib().orc_graph_from_csr_matrix(_p(indptr, _u64p), len(indptr) - 1,
                                               _p(indices, _u64p), _p(data, _f64p), len(data),
                                               _p(nw, _f64p), C.byref(h)))
        return cls(h)

    def info(self):
        n, e, ec = C.c_uint64(), C.c_uint64(), C.c_uint64()
        tw, loops = C.c_double(), C.c_int32()
        lib().orc_graph_info(self._h, C.byref(n), C.byref(e), C.byref(ec), C.byref(tw),
                             C.byref(loops))
        return dict(n=n.value, entries=e.value, edge_count=ec.value, total_weight=tw.value,
                    any_self_loops=bool(loops.value))

    @property
    def n(self):
        return self.info()["n"]

    def node_count(self):
        return self.n

    def edge_count(self):
        return self.info()["edge_count"]

    def total_weight(self):
        return self.info()["total_weight"]

    def arrays(self):
        i = self.info()
        ptr = np.zeros(i["n"] + 1, np.uint64)
        nbr = np.zeros(i["entries"], np.uint32)
        w = np.zeros(i["entries"], np.float32)
        nw = np.zeros(i["n"], np.float64)
        st = np.zeros(i["n"], np.float64)
        lib().orc_graph_arrays(self._h, _p(ptr, _u64p), _p(nbr, _u32p), _p(w, _f32p),
                               _p(nw, _f64p), _p(st, _f64p))
        return dict(ptr=ptr, nbr=nbr, w=w, node_w=nw, strength=st, **i)

    def strength(self, v):
        return float(self.arrays()["strength"][v])

    def validate_symmetry(self):
        _check(lib().orc_validate_symmetry(self._h))

    def aggregate(self, groups):
        g = np.ascontiguousarray(groups, dtype=np.uint64)
        h = C.c_void_p()
        _check(lib().orc_aggregate(self._h, _p(g, _u64p), len(g), C.byref(h)))
        return Graph(h)

    def partition_stats(self, memb):
        m = np.ascontiguousarray(memb, dtype=np.uint64)
        cap = int(m.max()) + 1 if len(m) else 0
        slots = C.c_uint64()
        size = np.zeros(cap, np.uint32)
        wt = np.zeros(cap, np.float64)
        st = np.zeros(cap, np.float64)
        inn = np.zeros(cap, np.float64)
        _check(lib().orc_partition_stats(self._h, _p(m, _u64p), len(m), C.byref(slots),
                                         _p(size, _u32p), _p(wt, _f64p), _p(st, _f64p),
                                         _p(inn, _f64p), cap))
        return dict(size=size, weight=wt, strength=st, internal=inn)

    def quality(self, memb, objective=RB, resolution=1.0):
        m = np.ascontiguousarray(memb, dtype=np.uint64)
        out = C.c_double()
        _check(lib().orc_quality(self._h, _p(m, _u64p), len(m), objective, resolution,
                                 C.byref(out)))
        return out.value

    def modularity(self, labels, resolution=1.0):
        m = np.ascontiguousarray(labels, dtype=np.uint64)
        out = C.c_double()
        _check(lib().orc_modularity(self._h, _p(m, _u64p), len(m), resolution, C.byref(out)))
        return out.value

    def local_move(self, memb, objective=RB, resolution=1.0, seed=0, max_cw=None):
        m = np.array(memb, dtype=np.uint64)
        gain = C.c_double()
        _check(lib().orc_local_move(self._h, _p(m, _u64p), len(m), objective, resolution, seed,
                                    0 if max_cw is None else 1, 0.0 if max_cw is None else max_cw,
                                    C.byref(gain)))
        return m, gain.value

    def refine(self, constraint, objective=RB, resolution=1.0, seed=0, max_cw=None,
               randomness=0.01):
        c = np.ascontiguousarray(constraint, dtype=np.uint32)
        out = np.zeros(len(c), np.uint64)
        _check(lib().orc_refine(self._h, _p(c, _u32p), len(c), objective, resolution, seed,
                                0 if max_cw is None else 1, 0.0 if max_cw is None else max_cw,
                                randomness, _p(out, _u64p)))
        return out

    def leiden(self, config: LeidenConfig | None = None, initial=None, **kw):
        cfg = config if config is not None else LeidenConfig.make(**kw)
        n = self.n
        labels = np.zeros(n, np.uint64)
        ncl = C.c_uint64()
        ini = None if initial is None else np.ascontiguousarray(initial, dtype=np.uint64)
        _check(lib().orc_leiden(self._h, C.byref(cfg), _p(ini, _u64p), _p(labels, _u64p),
                                C.byref(ncl)))
        return labels, ncl.value
