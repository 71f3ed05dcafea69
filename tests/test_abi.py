"""The C ABI library loads and exports every symbol include/sc_gpu.h declares.

Runs on the CPU: it only resolves symbols and calls the pure host helpers
(version, default config), never anything that touches a GPU.
"""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sc_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from sc_gpu import _lib
    return _lib.lib()


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("sc_graph_from_csr", "sc_graph_from_edges", "sc_leiden", "sc_leiden_from",
                     "sc_leiden_batch", "sc_modularity", "sc_quality", "sc_aggregate",
                     "sc_knn_gaussian", "sc_last_error_message"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    from sc_gpu import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_abi_version_and_default_config(lib):
    from sc_gpu import _lib
    assert lib.sc_abi_version() == 1
    c = _lib.LeidenConfigC()
    lib.sc_leiden_config_default(C.byref(c))
    # LeidenConfig::default (src/community_search/leiden/mod.rs:92-106)
    assert (c.objective, c.resolution, c.has_seed, c.seed) == (0, 1.0, 1, 42)
    assert (c.n_iterations, c.max_levels, c.tolerance) == (2, 64, 1e-9)
    assert (c.refine, c.refine_randomness, c.patience, c.has_max_community_weight) == (1, 0.01, 2, 0)


def test_python_config_matches_c_default():
    import sc_gpu
    from sc_gpu import _lib
    lib = _lib.lib()
    c = _lib.LeidenConfigC()
    lib.sc_leiden_config_default(C.byref(c))
    p = sc_gpu.LeidenConfig().to_c()
    for name, _ in _lib.LeidenConfigC._fields_:
        assert getattr(p, name) == getattr(c, name), name


def test_struct_layouts_match_header():
    from sc_gpu import _lib
    # sc_error_info: 1 int32 + padding, 4 u64, f64, 2 u64, 2 f64, 256 chars
    assert C.sizeof(_lib.ErrorInfo) == 8 + 4 * 8 + 8 + 2 * 8 + 2 * 8 + 256
    assert C.sizeof(_lib.LeidenConfigC) == 96
