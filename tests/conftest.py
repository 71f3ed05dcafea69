"""pytest configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a CUDA device and libsc_gpu.so; everything else runs on
the CPU (oracle vs golden vectors, host logic, ABI exports, gloo ranks).
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "single-clustering_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libsc_gpu.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")
