"""Learned warm start: an edge MLP trained on the GPU proposes an initial
membership for leiden_from (the `initial` of run_once,
src/community_search/leiden/mod.rs:207-220).

single-clustering has no learned component; this module adds one on top of
its warm-start hook. The network, its features and kernels are described in
include/sc_gpu.h (sc_mlp_*). Training and inference run in the library's own
CUDA kernels; nothing here computes on the host except bookkeeping.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import lib


def _check(rc, ctx):
    from . import _check as chk
    chk(rc, ctx)


def _ctx_labels(context):
    """(coarse, fine) host label arrays of a neighbouring-resolution context, or Nones."""
    if context is None:
        return None, None
    coarse, fine = context
    c = None if coarse is None else np.ascontiguousarray(coarse, np.uint64)
    f = None if fine is None else np.ascontiguousarray(fine, np.uint64)
    return c, f


def _p64(a):
    return None if a is None else a.ctypes.data_as(_lib.u64p)


def param_count() -> int:
    return int(lib().sc_mlp_param_count())


def feature_count() -> int:
    return int(lib().sc_mlp_feature_count())


class EdgeMlp:
    """Handle to a device-resident sc_mlp (parameters, Adam state, feature scaler)."""

    def __init__(self, seed: int = 0, *, device: int | None = None):
        self._ctx = _lib.context(device)
        self._h = C.c_void_p()
        _check(lib().sc_mlp_create(self._ctx.h, int(seed), C.byref(self._h)), self._ctx)

    def __del__(self):
        try:
            if self._h:
                lib().sc_mlp_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # state ----------------------------------------------------------------
    def params(self) -> np.ndarray:
        p = np.zeros(param_count(), np.float32)
        _check(lib().sc_mlp_get(self._ctx.h, self._h, p.ctypes.data_as(_lib.f32p), None, None), self._ctx)
        return p

    def scaler(self):
        """(means, inverse std) of the features, or None before the first fit."""
        s = np.zeros(2 * feature_count(), np.float32)
        has = C.c_int32()
        _check(lib().sc_mlp_get(self._ctx.h, self._h, None, s.ctypes.data_as(_lib.f32p), C.byref(has)), self._ctx)
        if not has.value:
            return None
        F = feature_count()
        return s[:F].copy(), s[F:].copy()

    def set_params(self, params=None, scaler=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        if p is not None and p.size != param_count():
            raise ValueError(f"expected {param_count()} parameters, got {p.size}")
        s = None
        if scaler is not None:
            s = np.ascontiguousarray(np.concatenate([scaler[0], scaler[1]]), np.float32)
        _check(lib().sc_mlp_set(self._ctx.h, self._h, None if p is None else p.ctypes.data_as(_lib.f32p),
                                None if s is None else s.ctypes.data_as(_lib.f32p)), self._ctx)

    # device work ------------------------------------------------------------
    def features(self, graph, resolution: float, context=None):
        """(features (M, F) float32, ei, ej) as the model sees them. `context` is
        (coarse, fine): the partitions found at a neighbouring lower and higher
        resolution (either may be None)."""
        cl, fl = _ctx_labels(context)
        cap = graph.entry_count()
        F = feature_count()
        feat = np.zeros((max(cap, 1), F), np.float32)
        ei = np.zeros(max(cap, 1), np.uint32)
        ej = np.zeros(max(cap, 1), np.uint32)
        M = C.c_uint64()
        _check(lib().sc_mlp_features(self._ctx.h, self._h, graph._h, float(resolution), _p64(cl), _p64(fl),
                                     feat.ctypes.data_as(_lib.f32p), ei.ctypes.data_as(_lib.u32p),
                                     ej.ctypes.data_as(_lib.u32p),
                                     cap, C.byref(M)), self._ctx)
        m = M.value
        return feat[:m], ei[:m], ej[:m]

    def train(self, graph, membership, resolution: float, epochs: int = 1, lr: float = 1e-2,
              return_grad: bool = False, context=None):
        """`epochs` Adam steps; returns the loss before the last step (and the gradient)."""
        m = np.ascontiguousarray(membership, np.uint64)
        cl, fl = _ctx_labels(context)
        loss = C.c_double()
        grad = np.zeros(param_count(), np.float32) if return_grad else None
        _check(lib().sc_mlp_train(self._ctx.h, self._h, graph._h, m.ctypes.data_as(_lib.u64p), len(m),
                                  float(resolution), _p64(cl), _p64(fl), int(epochs), float(lr), C.byref(loss),
                                  None if grad is None else grad.ctypes.data_as(_lib.f32p)), self._ctx)
        return (loss.value, grad) if return_grad else loss.value

    def propose(self, graph, resolution: float, threshold: float = 0.9, core_fraction: float = 1.0,
                return_prob: bool = False, context=None):
        """Initial membership: components of the confident edges (p > threshold)
        between core nodes (>= core_fraction of their edges confident)."""
        cl, fl = _ctx_labels(context)
        n = graph.node_count()
        labels = np.zeros(n, np.uint64)
        k = C.c_uint64()
        prob = np.zeros(max(graph.entry_count(), 1), np.float32) if return_prob else None
        _check(lib().sc_mlp_propose(self._ctx.h, self._h, graph._h, float(resolution), _p64(cl), _p64(fl),
                                    float(threshold), float(core_fraction), labels.ctypes.data_as(_lib.u64p),
                                    C.byref(k),
                                    None if prob is None else prob.ctypes.data_as(_lib.f32p),
                                    0 if prob is None else prob.size), self._ctx)
        if return_prob:
            return labels, k.value, prob
        return labels, k.value


@dataclass
class WarmStartResult:
    labels: np.ndarray
    n_clusters: int
    used_proposal: bool       # False: the plain singleton start won (fallback)
    q_warm: float
    q_plain: float | None
    sweeps_warm: int
    sweeps_plain: int | None
    ms_warm: float            # propose (host wall clock) + leiden_from (the library's device timing)
    ms_plain: float | None
    proposal_clusters: int
    ms_proposal: float | None = None  # the propose part of ms_warm (host wall clock)


def warm_start_leiden(model: EdgeMlp, graph, config, *, threshold: float = 0.9, core_fraction: float = 1.0,
                      verify: bool = True, tolerance: float = 1e-4, context=None,
                      warm_passes: int | None = 1) -> WarmStartResult:
    """leiden_from(model's proposal). With `verify`, the plain singleton start also
    runs and the proposal is kept only if its final modularity (for CPM: its CPM
    quality / total weight) is at least the plain one's minus `tolerance`;
    otherwise the plain result is returned.
    `context` is (coarse, fine), the partitions at the neighbouring lower and
    higher resolutions the model was trained to read. The warm run makes
    `warm_passes` passes (the proposal stands in for the first pass of a plain
    run, which takes the singleton start to a converged partition); None keeps
    config.n_iterations."""
    from . import leiden, leiden_from, modularity, quality, Rb
    is_rb = isinstance(config.objective, Rb)
    gamma = config.objective.resolution if is_rb else 1.0

    def score(labels):
        # the quantity the run optimises: modularity at gamma for RB; for CPM its
        # quality (Partition::from_membership then Cpm::quality) per unit of total
        # edge weight, the scale modularity has, so one tolerance serves both
        if is_rb:
            return modularity(graph, labels, gamma)
        return quality(graph, labels, config.objective) / max(graph.total_weight(), 1e-300)
    t0 = time.perf_counter()
    prop, kprop = model.propose(graph, gamma, threshold, core_fraction, context=context)
    t_prop = (time.perf_counter() - t0) * 1e3
    wcfg = config
    if warm_passes is not None:
        from dataclasses import replace
        wcfg = replace(config, n_iterations=int(warm_passes))
    warm = leiden_from(graph, wcfg, prop)
    sw = graph._ctx.run_stats()
    q_w = score(warm.labels())
    res = WarmStartResult(warm.labels(), warm.n_clusters(), True, q_w, None, sw["local_move_sweeps"], None,
                          t_prop + sw["ms_total"], None, kprop, t_prop)
    if not verify:
        return res
    plain = leiden(graph, config)
    sp = graph._ctx.run_stats()
    q_p = score(plain.labels())
    res.q_plain, res.sweeps_plain, res.ms_plain = q_p, sp["local_move_sweeps"], sp["ms_total"]
    if q_w < q_p - tolerance:
        res.labels, res.n_clusters, res.used_proposal = plain.labels(), plain.n_clusters(), False
    return res
