"""sc_gpu — single-clustering's Leiden hot path on B200, behind the reference API.

Mirrors single-clustering v0.7.0 (names, argument meaning and error
behaviour) over the C ABI of include/sc_gpu.h:

    CSRNetwork.from_edges / from_csr_parts / from_csr_matrix  (src/network/csr_network.rs)
    leiden(graph, LeidenConfig) -> Clustering                 (src/community_search/leiden/mod.rs)
    modularity(graph, labels, resolution)                     (.../leiden/objective.rs:221)
    Rb / Cpm objectives                                       (.../leiden/objective.rs:188-199)
    knn_gaussian(X, k, ...)                                   (src/neighborhood/mod.rs)

All computation runs in libsc_gpu.so on the GPU; nothing here computes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterable, Optional, Sequence, Union

import numpy as np

from . import _lib
from ._lib import context, lib

MAX_NODES = 0xFFFFFFFF  # csr_network.rs:36
NOISE = (1 << 64) - 1   # clustering.rs:8


# ---------------------------------------------------------------- errors
class ClusteringError(Exception):
    """ClusteringError (src/error.rs:7-68); `code` is the sc_status value."""

    code = 0

    def __init__(self, info: "_lib.ErrorInfo"):
        self.info = info
        super().__init__(info.message.decode("utf-8", errors="replace"))


class NodeIndexOutOfRange(ClusteringError):
    code = 1

    @property
    def node(self):
        return self.info.node

    @property
    def n_nodes(self):
        return self.info.n_nodes


class NonFiniteWeight(ClusteringError):
    code = 2

    @property
    def edge(self):
        return (self.info.edge_from, self.info.edge_to)


class NegativeWeight(ClusteringError):
    code = 3

    @property
    def edge(self):
        return (self.info.edge_from, self.info.edge_to)

    @property
    def weight(self):
        return self.info.weight


class InvalidNodeWeight(ClusteringError):
    code = 4

    @property
    def node(self):
        return self.info.node

    @property
    def weight(self):
        return self.info.weight


class NodeWeightLengthMismatch(ClusteringError):
    code = 5


class MembershipLengthMismatch(ClusteringError):
    code = 6


class InvalidConfig(ClusteringError):
    code = 7


class TooManyNodes(ClusteringError):
    code = 8


class InvalidCsr(ClusteringError):
    code = 9


class AsymmetricGraph(ClusteringError):
    code = 10

    @property
    def degree_sum(self):
        return self.info.degree_sum

    @property
    def expected(self):
        return self.info.expected


class DeviceError(ClusteringError):
    """Failures the Rust API has no variant for (CUDA, allocation, timeout, ...)."""


_BY_CODE = {cls.code: cls for cls in (NodeIndexOutOfRange, NonFiniteWeight, NegativeWeight,
                                      InvalidNodeWeight, NodeWeightLengthMismatch,
                                      MembershipLengthMismatch, InvalidConfig, TooManyNodes,
                                      InvalidCsr, AsymmetricGraph)}


def _check(rc: int, ctx):
    if rc != 0:
        info = ctx.error_info()
        cls = _BY_CODE.get(rc, DeviceError)
        err = cls(info)
        err.status = rc
        raise err


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


# ---------------------------------------------------------------- config
@dataclass(frozen=True)
class Rb:
    """Reichardt-Bornholdt configuration model (objective.rs:66-125)."""
    resolution: float = 1.0


@dataclass(frozen=True)
class Cpm:
    """Constant Potts Model (objective.rs:127-184)."""
    resolution: float = 0.05


ObjectiveKind = Union[Rb, Cpm]


@dataclass
class LeidenConfig:
    """LeidenConfig (src/community_search/leiden/mod.rs:49-106)."""
    objective: ObjectiveKind = field(default_factory=Rb)
    seed: Optional[int] = 42
    n_iterations: int = 2
    max_levels: int = 64
    tolerance: float = 1e-9
    refine: bool = True
    refine_randomness: float = 0.01
    patience: int = 2
    max_community_weight: Optional[float] = None

    @classmethod
    def with_resolution(cls, resolution: float) -> "LeidenConfig":
        return cls(objective=Rb(resolution))

    def to_c(self) -> _lib.LeidenConfigC:
        c = _lib.LeidenConfigC()
        c.objective = 0 if isinstance(self.objective, Rb) else 1
        c.resolution = float(self.objective.resolution)
        c.has_seed = 0 if self.seed is None else 1
        c.seed = 0 if self.seed is None else int(self.seed) & ((1 << 64) - 1)
        c.n_iterations = int(self.n_iterations)
        c.max_levels = int(self.max_levels)
        c.tolerance = float(self.tolerance)
        c.refine = 1 if self.refine else 0
        c.refine_randomness = float(self.refine_randomness)
        c.patience = int(self.patience)
        c.has_max_community_weight = 0 if self.max_community_weight is None else 1
        c.max_community_weight = 0.0 if self.max_community_weight is None else float(
            self.max_community_weight)
        return c


# ---------------------------------------------------------------- result
class Clustering:
    """Clustering (src/clustering.rs:11-108)."""

    def __init__(self, labels: np.ndarray, n_clusters: int):
        self._labels = labels
        self._n = int(n_clusters)

    def labels(self) -> np.ndarray:
        return self._labels

    def n_clusters(self) -> int:
        return self._n

    def __len__(self):
        return len(self._labels)

    def is_empty(self) -> bool:
        return len(self._labels) == 0

    def cluster_sizes(self) -> list:
        return np.bincount(self._labels.astype(np.int64), minlength=self._n).tolist()

    def into_labels(self) -> np.ndarray:
        return self._labels

    def __eq__(self, other):
        return isinstance(other, Clustering) and self._n == other._n and np.array_equal(
            self._labels, other._labels)


# ---------------------------------------------------------------- graph
class CSRNetwork:
    """A device-resident CSRNetwork (src/network/csr_network.rs:62-69)."""

    def __init__(self, handle: C.c_void_p, ctx):
        self._h = handle
        self._ctx = ctx

    def __del__(self):
        try:
            if self._h:
                lib().sc_graph_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # constructors -------------------------------------------------------
    @classmethod
    def from_edges(cls, n_nodes: int, edges: Iterable, *, device: int | None = None):
        """from_edges (csr_network.rs:104-109); edges are (u, v, w) tuples or an (m, 3) array."""
        return cls._from_edges(n_nodes, edges, None, device)

    @classmethod
    def from_edges_with_node_weights(cls, edges: Iterable, node_weights: Sequence[float], *,
                                     device: int | None = None):
        nw = np.ascontiguousarray(node_weights, dtype=np.float64)
        return cls._from_edges(len(nw), edges, nw, device)

    @classmethod
    def from_edge_arrays(cls, n_nodes: int, src, dst, w, node_weights=None, *, device=None):
        src = np.ascontiguousarray(src, dtype=np.uint64)
        dst = np.ascontiguousarray(dst, dtype=np.uint64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        nw = None if node_weights is None else np.ascontiguousarray(node_weights, np.float64)
        ctx = context(device)
        h = C.c_void_p()
        _check(lib().sc_graph_from_edges(ctx.h, int(n_nodes), _ptr(src, _lib.u64p), _ptr(dst, _lib.u64p),
                                         _ptr(w, _lib.f64p), len(src), _ptr(nw, _lib.f64p),
                                         C.byref(h)), ctx)
        return cls(h, ctx)

    @classmethod
    def _from_edges(cls, n_nodes, edges, nw, device):
        if isinstance(edges, np.ndarray) and edges.ndim == 2:
            src, dst, w = edges[:, 0], edges[:, 1], edges[:, 2]
        else:
            edges = list(edges)
            src = [int(e[0]) for e in edges]
            dst = [int(e[1]) for e in edges]
            w = [float(e[2]) for e in edges]
        return cls.from_edge_arrays(n_nodes, np.array(src, dtype=np.uint64),
                                    np.array(dst, dtype=np.uint64), np.array(w, dtype=np.float64),
                                    nw, device=device)

    @classmethod
    def from_csr_parts(cls, node_ptrs, neighbors, weights, node_weights=None, *, device=None):
        """from_csr_parts (csr_network.rs:185-256)."""
        ptrs = np.ascontiguousarray(node_ptrs, dtype=np.uint64)
        nbrs = np.ascontiguousarray(neighbors, dtype=np.uint32)
        w = np.ascontiguousarray(weights, dtype=np.float32)
        nw = None if node_weights is None else np.ascontiguousarray(node_weights, np.float64)
        ctx = context(device)
        h = C.c_void_p()
        _check(lib().sc_graph_from_csr(ctx.h, _ptr(ptrs, _lib.u64p), len(ptrs), _ptr(nbrs, _lib.u32p),
                                       len(nbrs), _ptr(w, _lib.f32p), len(w), _ptr(nw, _lib.f64p),
                                       0 if nw is None else len(nw), C.byref(h)), ctx)
        return cls(h, ctx)

    @classmethod
    def from_csr_parts_device(cls, node_ptrs, neighbors, weights, node_weights=None, *, device=None):
        """from_csr_parts on torch CUDA tensors already on the device (no host round trip)."""
        ctx = context(device)
        h = C.c_void_p()
        nwp = None if node_weights is None else node_weights.data_ptr()
        _check(lib().sc_graph_from_csr_device(ctx.h, node_ptrs.data_ptr(), node_ptrs.numel(),
                                              neighbors.data_ptr(), neighbors.numel(),
                                              weights.data_ptr(), weights.numel(), nwp,
                                              0 if node_weights is None else node_weights.numel(),
                                              C.byref(h)), ctx)
        return cls(h, ctx)

    @classmethod
    def from_csr_matrix(cls, indptr, indices, data, node_weights=None, *, device=None):
        """from_csr_matrix (csr_network.rs:360-391): reads the upper triangle only."""
        indptr = np.ascontiguousarray(indptr, dtype=np.uint64)
        indices = np.ascontiguousarray(indices, dtype=np.uint64)
        data = np.ascontiguousarray(data, dtype=np.float64)
        n = len(indptr) - 1
        nw = None if node_weights is None else np.ascontiguousarray(node_weights, np.float64)
        if nw is not None and len(nw) != n:
            raise NodeWeightLengthMismatch(_mismatch_info(5, len(nw), n,
                                                          "node weight vector has length {got}, expected {exp}"))
        ctx = context(device)
        h = C.c_void_p()
        _check(lib().sc_graph_from_csr_matrix(ctx.h, _ptr(indptr, _lib.u64p), n, _ptr(indices, _lib.u64p),
                                              _ptr(data, _lib.f64p), len(data), _ptr(nw, _lib.f64p),
                                              C.byref(h)), ctx)
        return cls(h, ctx)

    # accessors ----------------------------------------------------------
    def _info(self):
        n, e, ec = C.c_uint64(), C.c_uint64(), C.c_uint64()
        tw, loops = C.c_double(), C.c_int32()
        lib().sc_graph_info(self._h, C.byref(n), C.byref(e), C.byref(ec), C.byref(tw), C.byref(loops))
        return n.value, e.value, ec.value, tw.value, bool(loops.value)

    def node_count(self) -> int:
        return self._info()[0]

    def entry_count(self) -> int:
        return self._info()[1]

    def edge_count(self) -> int:
        return self._info()[2]

    def total_weight(self) -> float:
        return self._info()[3]

    def has_self_loops(self) -> bool:
        return self._info()[4]

    def set_embedding(self, X) -> None:
        """Attaches the kNN embedding the graph was built from (node_count x d
        points): the learned warm start reads the edge's length in a fixed
        16-component projection of it, relative to the endpoints' local scale."""
        X = np.ascontiguousarray(X, np.float32)
        if X.ndim != 2:
            raise ValueError("embedding must be a 2-D array (nodes x dims)")
        _check(lib().sc_graph_set_embedding(self._ctx.h, self._h, _ptr(X, _lib.f32p), X.shape[0], X.shape[1]),
               self._ctx)

    def to_csr_parts(self):
        n, e, *_ = self._info()
        ptr = np.zeros(n + 1, np.uint64)
        nbr = np.zeros(e, np.uint32)
        w = np.zeros(e, np.float32)
        _check(lib().sc_graph_copy_csr(self._ctx.h, self._h, _ptr(ptr, _lib.u64p), _ptr(nbr, _lib.u32p),
                                       _ptr(w, _lib.f32p)), self._ctx)
        return ptr, nbr, w

    def node_weights(self) -> np.ndarray:
        n = self.node_count()
        nw = np.zeros(n, np.float64)
        _check(lib().sc_graph_copy_node_data(self._ctx.h, self._h, _ptr(nw, _lib.f64p), None), self._ctx)
        return nw

    def strengths(self) -> np.ndarray:
        n = self.node_count()
        st = np.zeros(n, np.float64)
        _check(lib().sc_graph_copy_node_data(self._ctx.h, self._h, None, _ptr(st, _lib.f64p)), self._ctx)
        return st

    def strength(self, node: int) -> float:
        return float(self.strengths()[node])

    def node_weight(self, node: int) -> float:
        return float(self.node_weights()[node])

    def degree(self, node: int) -> int:
        ptr, _, _ = self.to_csr_parts()
        return int(ptr[node + 1] - ptr[node])

    def neighbors(self, node: int):
        ptr, nbr, w = self.to_csr_parts()
        s, e = int(ptr[node]), int(ptr[node + 1])
        return [(int(u), float(x)) for u, x in zip(nbr[s:e], w[s:e])]

    def self_loop_weight(self, node: int) -> float:
        for u, x in self.neighbors(node):
            if u == node:
                return x
        return 0.0

    def edge_weight(self, a: int, b: int):
        for u, x in self.neighbors(a):
            if u == b:
                return x
        return None

    def validate_symmetry(self):
        _check(lib().sc_graph_validate_symmetry(self._ctx.h, self._h), self._ctx)

    def aggregate(self, groups) -> "CSRNetwork":
        """aggregate(&VectorGrouping::from_assignments(groups)) (csr_network.rs:516-608)."""
        g = np.ascontiguousarray(groups, dtype=np.uint64)
        h = C.c_void_p()
        _check(lib().sc_aggregate(self._ctx.h, self._h, _ptr(g, _lib.u64p), len(g), C.byref(h)), self._ctx)
        return CSRNetwork(h, self._ctx)

    def partition_stats(self, membership):
        """Partition::from_membership aggregates (partition.rs:75-112) per slot."""
        m = np.ascontiguousarray(membership, dtype=np.uint64)
        cap = int(m.max()) + 1 if len(m) else 0
        slots = C.c_uint64()
        size = np.zeros(cap, np.uint32)
        wt = np.zeros(cap, np.float64)
        st = np.zeros(cap, np.float64)
        inn = np.zeros(cap, np.float64)
        _check(lib().sc_partition_stats(self._ctx.h, self._h, _ptr(m, _lib.u64p), len(m), C.byref(slots),
                                        _ptr(size, _lib.u32p), _ptr(wt, _lib.f64p), _ptr(st, _lib.f64p),
                                        _ptr(inn, _lib.f64p), cap), self._ctx)
        return dict(size=size, weight=wt, strength=st, internal=inn)

    def __str__(self):
        n, _, ec, tw, _ = self._info()
        dens = ec / (n * (n - 1) / 2) if n > 1 else 0.0
        return f"CSRNetwork({n} nodes, {ec} edges, total_weight: {tw}, density: {dens:.4f})"


def _mismatch_info(code, got, exp, fmt):
    i = _lib.ErrorInfo()
    i.code = code
    i.got = got
    i.expected_len = exp
    i.message = fmt.format(got=got, exp=exp).encode()
    return i


# ---------------------------------------------------------------- algorithms
def leiden(graph: CSRNetwork, config: LeidenConfig | None = None) -> Clustering:
    """leiden(&graph, &config) (src/community_search/leiden/mod.rs:168-204)."""
    return leiden_from(graph, config, None)


def leiden_from(graph: CSRNetwork, config: LeidenConfig | None, initial) -> Clustering:
    """leiden starting from `initial` labels (the `initial` of run_once, mod.rs:214-220)."""
    cfg = (config or LeidenConfig()).to_c()
    n = graph.node_count()
    labels = np.zeros(n, np.uint64)
    ncl = C.c_uint64()
    ini = None if initial is None else np.ascontiguousarray(initial, dtype=np.uint64)
    ctx = graph._ctx
    _check(lib().sc_leiden_from(ctx.h, graph._h, C.byref(cfg), _ptr(ini, _lib.u64p),
                                0 if ini is None else len(ini), _ptr(labels, _lib.u64p), C.byref(ncl)), ctx)
    return Clustering(labels, ncl.value)


def leiden_batch(graphs: Sequence[CSRNetwork], configs: Sequence[LeidenConfig], warm_from=None,
                 n_streams: int = 0, union: bool = False, max_union_entries: int = 0) -> list:
    """Many leiden() runs in one call.

    union=False: concurrently on `n_streams` worker streams (sc_leiden_batch_ex).
    union=True: as batched device work over disjoint unions of the instances'
    graphs (sc_leiden_batch_union): every launch covers all instances whose
    warm start is done; labels equal the separate runs' inside the exact
    summation regime.

    warm_from[i] = j (j < i) starts instance i from instance j's labels (leiden
    with `initial`); -1 starts from singletons."""
    count = len(graphs)
    if count == 0:
        return []
    ctx = graphs[0]._ctx
    sizes = [g.node_count() for g in graphs]
    offs = np.zeros(count, np.uint64)
    offs[1:] = np.cumsum(sizes)[:-1]
    labels = np.zeros(int(sum(sizes)), np.uint64)
    ncl = np.zeros(count, np.uint64)
    harr = (C.c_void_p * count)(*[g._h for g in graphs])
    carr = (_lib.LeidenConfigC * count)(*[c.to_c() for c in configs])
    wf = None
    if warm_from is not None:
        wf = np.ascontiguousarray(warm_from, dtype=np.int64)
    wfp = None if wf is None else wf.ctypes.data_as(C.POINTER(C.c_int64))
    if union:
        _check(lib().sc_leiden_batch_union(ctx.h, harr, carr, count, wfp, _ptr(offs, _lib.u64p),
                                           _ptr(labels, _lib.u64p), _ptr(ncl, _lib.u64p),
                                           int(max_union_entries)), ctx)
    else:
        _check(lib().sc_leiden_batch_ex(ctx.h, harr, carr, count, wfp, _ptr(offs, _lib.u64p),
                                        _ptr(labels, _lib.u64p), _ptr(ncl, _lib.u64p), int(n_streams)), ctx)
    out = []
    for i in range(count):
        s0 = int(offs[i])
        out.append(Clustering(labels[s0:s0 + sizes[i]].copy(), int(ncl[i])))
    return out


def sweep_plan(resolutions: Sequence[float], seeds: Sequence[int], objective=Rb, warm_start: bool = True,
               base: LeidenConfig | None = None, split: int = 1, warm_passes: int | None = 1):
    """Configs and warm-start links of a resolution x seed sweep.

    Instances are ordered seed-major with resolutions descending; with warm_start
    each instance starts from the previous (finer) resolution's result of the
    same seed, so a chain coarsens a partition instead of rebuilding it. With
    split = k each seed's chain is cut into k contiguous pieces: the first piece
    starts from singletons, the head of every other piece from the first
    instance of the seed (the finest resolution), so k pieces per seed run
    concurrently. A warm-started instance runs `warm_passes` passes (its start
    stands in for the first pass of a plain run, which takes a singleton start
    to a converged partition); None keeps the base config's n_iterations.
    Returns (configs, warm_from, keys)."""
    base = base or LeidenConfig()
    res = sorted(resolutions, reverse=True)
    split = max(1, min(int(split), len(res))) if res else 1
    bounds = [round(i * len(res) / split) for i in range(split + 1)]
    heads = set(bounds[:-1])
    configs, warm, keys = [], [], []
    for s in seeds:
        first = len(configs)
        for j, r in enumerate(res):
            fields = {**base.__dict__, "objective": objective(r), "seed": int(s)}
            if warm_start and j > 0 and warm_passes is not None:
                fields["n_iterations"] = int(warm_passes)
            configs.append(LeidenConfig(**fields))
            if not warm_start or j == 0:
                warm.append(-1)
            elif j in heads:
                warm.append(first)
            else:
                warm.append(len(configs) - 2)
            keys.append((float(r), int(s)))
    return configs, warm, keys


def leiden_sweep(graph: CSRNetwork, resolutions, seeds, objective=Rb, warm_start: bool = True,
                 n_streams: int = 0, base: LeidenConfig | None = None, split: int = 1,
                 warm_passes: int | None = 1, union: bool = False, max_union_entries: int = 0) -> dict:
    """Resolution x seed sweep on one graph: {(resolution, seed): Clustering}."""
    configs, warm, keys = sweep_plan(resolutions, seeds, objective, warm_start, base, split, warm_passes)
    res = leiden_batch([graph] * len(configs), configs, warm if warm_start else None, n_streams, union,
                       max_union_entries)
    return dict(zip(keys, res))


def modularity(graph: CSRNetwork, labels, resolution: float = 1.0) -> float:
    """modularity (src/community_search/leiden/objective.rs:221-244)."""
    lab = np.ascontiguousarray(labels, dtype=np.uint64)
    out = C.c_double()
    _check(lib().sc_modularity(graph._ctx.h, graph._h, _ptr(lab, _lib.u64p), len(lab), float(resolution),
                               C.byref(out)), graph._ctx)
    return out.value


def quality(graph: CSRNetwork, membership, objective: ObjectiveKind = Rb()) -> float:
    """Rb::quality / Cpm::quality of Partition::from_membership (objective.rs:108-178)."""
    m = np.ascontiguousarray(membership, dtype=np.uint64)
    out = C.c_double()
    kind = 0 if isinstance(objective, Rb) else 1
    _check(lib().sc_quality(graph._ctx.h, graph._h, _ptr(m, _lib.u64p), len(m), kind,
                            float(objective.resolution), C.byref(out)), graph._ctx)
    return out.value


def get_tuning(device: int | None = None) -> dict:
    """The decide-kernel routing of this thread's context on `device`."""
    t = _lib.Tuning()
    ctx = context(device)
    _check(lib().sc_get_tuning(ctx.h, C.byref(t)), ctx)
    return {name: getattr(t, name) for name, _ in _lib.Tuning._fields_}


def set_tuning(tuning: dict, device: int | None = None) -> None:
    t = _lib.Tuning()
    lib().sc_tuning_default(C.byref(t))
    for k, v in tuning.items():
        setattr(t, k, int(v))
    ctx = context(device)
    _check(lib().sc_set_tuning(ctx.h, C.byref(t)), ctx)


def autotune(graph: CSRNetwork, config: LeidenConfig | None = None) -> dict:
    """Times the first Leiden level under candidate routings on `graph`, keeps
    the fastest on the graph's context; returns it with the timings (ms)."""
    cfg = (config or LeidenConfig()).to_c()
    t = _lib.Tuning()
    best, default = C.c_double(), C.c_double()
    k = C.c_uint32()
    ctx = graph._ctx
    _check(lib().sc_autotune(ctx.h, graph._h, C.byref(cfg), C.byref(t), C.byref(best), C.byref(default),
                             C.byref(k)), ctx)
    out = {name: getattr(t, name) for name, _ in _lib.Tuning._fields_}
    out.update(ms_chosen=best.value, ms_default=default.value, candidates=k.value)
    return out


def last_run_stats(device: int | None = None) -> dict:
    return context(device).run_stats()


__all__ = [
    "CSRNetwork", "LeidenConfig", "Rb", "Cpm", "ObjectiveKind", "Clustering", "leiden", "leiden_from",
    "leiden_batch", "modularity", "quality", "ClusteringError", "NodeIndexOutOfRange", "NonFiniteWeight",
    "NegativeWeight", "InvalidNodeWeight", "NodeWeightLengthMismatch", "MembershipLengthMismatch",
    "InvalidConfig", "TooManyNodes", "InvalidCsr", "AsymmetricGraph", "DeviceError", "MAX_NODES", "NOISE",
    "last_run_stats", "context", "sweep_plan", "leiden_sweep", "get_tuning", "set_tuning", "autotune",
]


# ---------------------------------------------------------------- kNN graph builder
SIGMA_MEDIAN, SIGMA_KTH = 0, 1
SYM_LOWER_ID, SYM_UNION = 0, 1
KNN_FP32, KNN_BF16, KNN_FP8 = 0, 1, 2


class NeighborResult:
    """NeighborResult (src/neighborhood/mod.rs:29-34): k+1 neighbours per row
    (self first) with their distances, and the connectivities CSR."""

    def __init__(self, index, distances, conn_ptrs, conn_nbrs, conn_w, graph=None):
        self.index = index
        self.distances = distances
        self.conn_ptrs = conn_ptrs
        self.conn_nbrs = conn_nbrs
        self.conn_w = conn_w
        self.graph = graph


def knn_gaussian(X, k: int, *, sigma: int = SIGMA_MEDIAN, sym: int = SYM_LOWER_ID,
                 precision: int = KNN_BF16, squared: bool = False, build_graph: bool = False,
                 device: int | None = None) -> NeighborResult:
    """knn_arrayd_* (neighborhood/mod.rs:51-202, :359-578) with an exact search.

    Defaults follow the reference: sigma = median neighbour distance, pairs
    emitted from the lower id only. `squared=True` mirrors the kd-tree path
    (squared distances returned, sigma = sqrt(median d^2))."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, d = X.shape
    ctx = context(device)
    opts = _lib.KnnOpts()
    lib().sc_knn_opts_default(C.byref(opts))
    opts.sigma, opts.sym, opts.precision, opts.squared_kiddo = sigma, sym, precision, int(squared)
    # outputs are written by the library in full: no zero fill. The entry
    # arrays are sized for the most entries possible (2 n k) and returned as
    # views of their first nnz; the unwritten tail is never touched, so it
    # takes no memory, and no copy is made.
    idx = np.empty((n, k + 1), np.uint32)
    dist = np.empty((n, k + 1), np.float32)
    cap = 2 * n * k
    ptrs = np.empty(n + 1, np.uint64)
    nbrs = np.empty(cap, np.uint32)
    w = np.empty(cap, np.float32)
    nnz = C.c_uint64()
    gh = C.c_void_p()
    _check(lib().sc_knn_gaussian(ctx.h, _ptr(X, _lib.f32p), n, d, k, C.byref(opts), _ptr(idx, _lib.u32p),
                                 _ptr(dist, _lib.f32p), _ptr(ptrs, _lib.u64p), _ptr(nbrs, _lib.u32p),
                                 _ptr(w, _lib.f32p), cap, C.byref(nnz),
                                 C.byref(gh) if build_graph else None), ctx)
    m = nnz.value
    graph = CSRNetwork(gh, ctx) if build_graph else None
    return NeighborResult(idx, dist, ptrs, nbrs[:m], w[:m], graph)


def set_knn_clusters(clusters: int, device: int | None = None) -> None:
    """Point clusters of the exact pruned kNN search (sc_set_knn_clusters):
    0 picks a count from n, 1 scans every point tile."""
    ctx = context(device)
    _check(lib().sc_set_knn_clusters(ctx.h, int(clusters)), ctx)


def knn_autotune(X, k: int, *, precision: int = KNN_BF16, device: int | None = None) -> dict:
    """Times the exact kNN search of X under candidate cluster counts (1 = full
    scan) and keeps the fastest on this thread's context (sc_knn_autotune)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, d = X.shape
    ctx = context(device)
    opts = _knn_opts(precision=precision)
    chosen, nc = C.c_uint32(), C.c_uint32()
    ms_c, ms_f = C.c_double(), C.c_double()
    _check(lib().sc_knn_autotune(ctx.h, _ptr(X, _lib.f32p), n, d, k, C.byref(opts), C.byref(chosen),
                                 C.byref(ms_c), C.byref(ms_f), C.byref(nc)), ctx)
    return {"clusters": chosen.value, "ms_chosen": ms_c.value, "ms_full": ms_f.value, "candidates": nc.value}


def knn_last_stats(device: int | None = None) -> dict:
    """Counters of the last kNN search on this thread's context: clusters,
    (query group, point tile) pairs scanned and those of a full scan."""
    ctx = context(device)
    st = _lib.KnnStats()
    _check(lib().sc_knn_last_stats(ctx.h, C.byref(st)), ctx)
    return {name: getattr(st, name) for name, _ in _lib.KnnStats._fields_}


def _knn_opts(sigma=SIGMA_MEDIAN, sym=SYM_LOWER_ID, precision=KNN_BF16, squared=False):
    opts = _lib.KnnOpts()
    lib().sc_knn_opts_default(C.byref(opts))
    opts.sigma, opts.sym, opts.precision, opts.squared_kiddo = sigma, sym, precision, int(squared)
    return opts


def knn_search(X, k: int, q_begin: int, q_end: int, *, precision: int = KNN_BF16, device: int | None = None):
    """The k+1 nearest points (self first) of the query rows [q_begin, q_end) of X
    among all rows: (index uint32 (q, k+1), squared distances float32 (q, k+1)).
    One shard of a build split by query rows (sc_knn_search)."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, d = X.shape
    ctx = context(device)
    opts = _knn_opts(precision=precision)
    nq = max(int(q_end) - int(q_begin), 0)
    idx = np.zeros((nq, k + 1), np.uint32)
    d2 = np.zeros((nq, k + 1), np.float32)
    _check(lib().sc_knn_search(ctx.h, _ptr(X, _lib.f32p), n, d, k, int(q_begin), int(q_end), C.byref(opts),
                               _ptr(idx, _lib.u32p), _ptr(d2, _lib.f32p)), ctx)
    return idx, d2


def knn_connectivities(index, d2, *, sigma: int = SIGMA_MEDIAN, sym: int = SYM_LOWER_ID, squared: bool = False,
                       build_graph: bool = False, device: int | None = None) -> NeighborResult:
    """Connectivities from the gathered (n, k+1) lists of knn_search
    (sc_knn_connectivities); distances in the result follow `squared`."""
    index = np.ascontiguousarray(index, dtype=np.uint32)
    d2 = np.ascontiguousarray(d2, dtype=np.float32)
    n, k1 = index.shape
    k = k1 - 1
    ctx = context(device)
    opts = _knn_opts(sigma, sym, KNN_BF16, squared)
    cap = 2 * n * k
    ptrs = np.empty(n + 1, np.uint64)  # written in full by the library (see knn_gaussian)
    nbrs = np.empty(max(cap, 1), np.uint32)
    w = np.empty(max(cap, 1), np.float32)
    nnz = C.c_uint64()
    gh = C.c_void_p()
    _check(lib().sc_knn_connectivities(ctx.h, _ptr(index, _lib.u32p), _ptr(d2, _lib.f32p), n, k, C.byref(opts),
                                       _ptr(ptrs, _lib.u64p), _ptr(nbrs, _lib.u32p), _ptr(w, _lib.f32p), cap,
                                       C.byref(nnz), C.byref(gh) if build_graph else None), ctx)
    m = nnz.value
    dist = d2 if squared else np.sqrt(d2)
    return NeighborResult(index, dist, ptrs, nbrs[:m], w[:m], CSRNetwork(gh, ctx) if build_graph else None)


__all__ += ["knn_search", "knn_connectivities"]
__all__ += ["knn_gaussian", "NeighborResult", "SIGMA_MEDIAN", "SIGMA_KTH", "SYM_LOWER_ID", "SYM_UNION",
            "KNN_FP32", "KNN_BF16", "KNN_FP8"]
