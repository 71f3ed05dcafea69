"""Regenerates the golden fixtures in this folder from single-clustering's own
test data. Runs only where the reference source tree is present (it is not on
the GPU machines, which use the committed outputs).

Outputs
  karate.json                 edge list of src/testdata.rs:8-23 and the known
                              optimum labelling of src/testdata.rs:31-36
  leidenalg_reference.json.gz tests/fixtures/leidenalg_reference.json verbatim
                              (10 graphs, 160 cases: leidenalg quality and
                              igraph modularity of a given membership)

Usage: python tests/golden/gen_golden.py /path/to/single-clustering
"""
import gzip
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_karate(testdata_rs: str):
    body = testdata_rs.split("const E: &[(usize, usize)] = &[", 1)[1].split("];", 1)[0]
    edges = [(int(a), int(b)) for a, b in re.findall(r"\((\d+),\s*(\d+)\)", body)]
    opt = testdata_rs.split("pub fn karate_optimum()", 1)[1].split("vec![", 1)[1].split("]", 1)[0]
    optimum = [int(x) for x in re.findall(r"\d+", opt)]
    return edges, optimum


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: gen_golden.py /path/to/single-clustering (the reference source tree)")
    ref = sys.argv[1]
    with open(os.path.join(ref, "src", "testdata.rs")) as f:
        edges, optimum = parse_karate(f.read())
    assert len(edges) == 78 and len(optimum) == 34, (len(edges), len(optimum))
    with open(os.path.join(HERE, "karate.json"), "w") as f:
        json.dump({"source": "src/testdata.rs:8-36", "n_nodes": 34, "edges": edges,
                   "optimum": optimum, "optimum_modularity": 0.4198}, f)
    src = os.path.join(ref, "tests", "fixtures", "leidenalg_reference.json")
    with open(src, "rb") as f:
        raw = f.read()
    json.loads(raw)  # must parse
    with open(os.path.join(HERE, "leidenalg_reference.json.gz"), "wb") as f:
        f.write(gzip.compress(raw, mtime=0))
    print("wrote karate.json and leidenalg_reference.json.gz")


if __name__ == "__main__":
    main()
