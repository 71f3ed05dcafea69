"""The real-data harness (sc_gpu.real_data, examples/real_data.rs): its export
reader, its partition-agreement scores (checked against scikit-learn's), and one
GPU run on a synthetic export in the reference's format."""
import json

import numpy as np
import pytest

from sc_gpu import real_data as rd


def test_ari_and_nmi_match_scikit_learn():
    from sklearn.metrics import adjusted_rand_score, normalized_mutual_info_score
    rng = np.random.default_rng(0)
    for n, ka, kb in ((10, 2, 3), (200, 5, 5), (1000, 20, 7), (50, 1, 4)):
        a = rng.integers(0, ka, n)
        b = rng.integers(0, kb, n)
        assert abs(rd.adjusted_rand_index(a, b) - adjusted_rand_score(a, b)) < 1e-12
        assert abs(rd.nmi(a, b) - normalized_mutual_info_score(a, b)) < 1e-12
    a = np.array([0, 0, 1, 1, 2, 2])
    assert rd.adjusted_rand_index(a, 5 - a) == 1.0  # relabelling changes nothing
    assert abs(rd.nmi(a, 5 - a) - 1.0) < 1e-12
    assert rd.adjusted_rand_index([], []) == 1.0 and rd.nmi([], []) == 1.0


def _write_export(path, ptr, nbr, w, reference, n):
    np.asarray(ptr, "<u8").tofile(path / "indptr.bin")
    np.asarray(nbr, "<u4").tofile(path / "indices.bin")
    np.asarray(w, "<f4").tofile(path / "data.bin")
    meta = {"dataset": "synthetic", "n_cells": n, "n_entries": int(len(nbr)), "n_neighbors": 0, "scanpy": "none"}
    (path / "meta.json").write_text(json.dumps(meta))
    (path / "reference.json").write_text(json.dumps(reference))


def test_export_reader_round_trip(tmp_path):
    ptr = [0, 2, 3, 4]
    nbr = [1, 2, 0, 0]
    w = [0.5, 1.5, 0.5, 1.5]
    ref = {"resolutions": {"1.0": {"labels": [0, 0, 1], "n_clusters": 2, "seconds": 0.1}}}
    _write_export(tmp_path, ptr, nbr, w, ref, 3)
    meta, reference, p, i, d = rd.load_export(str(tmp_path))
    assert meta["n_cells"] == 3 and reference == ref
    assert p.dtype == np.uint64 and list(p) == ptr
    assert i.dtype == np.uint32 and list(i) == nbr
    assert d.dtype == np.float32 and list(d) == w


@pytest.mark.gpu
def test_harness_on_a_synthetic_export(tmp_path):
    import sc_gpu
    from sc_gpu import synth
    n = 3000
    src, dst, w, truth = synth.planted_partition(n, 10, 8, 2, 3)
    g = sc_gpu.CSRNetwork.from_edge_arrays(n, src, dst, w)
    ptr, nbr, ww = g.to_csr_parts()
    truth = [int(t) for t in truth]
    ref = {"resolutions": {k: {"labels": truth, "n_clusters": 10, "seconds": 0.5} for k in ("0.5", "1.0")},
           "annotation": {"name": "planted", "categories": list(range(10)), "labels": truth}}
    _write_export(tmp_path, ptr, nbr, ww, ref, n)
    lines = []
    rows = rd.run(str(tmp_path), out=lines.append)
    assert [r["resolution"] for r in rows] == [0.5, 1.0]
    for r in rows:
        assert r["ari"] > 0.9 and r["nmi"] > 0.9, r
        assert r["ours_q"] >= r["scanpy_q"] - 1e-3
        assert r["ari_annotation"] == r["ari"]
    assert any(line.startswith("best agreement with author cell types") for line in lines)
    assert "exhaustive symmetry check: OK" in lines
