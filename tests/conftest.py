"""Shared test setup: the gpu marker, paths, and graph fixtures.

CPU tests (-m "not gpu") cover the oracle against the reference's binaries and
the committed golden fixtures, the generators, the host logic and the C ABI
exports.  GPU tests (-m gpu) compare the CUDA engine with the oracle."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402


os.environ.setdefault("IPG_MAX_SUPERSTEPS", "20000")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (runs the CUDA engine)")


def have_gpu():
    try:
        import ipregel_b200 as ip
        ip.device_info()
        return True
    except Exception:
        return False


def small_graphs():
    """Hand-made graphs covering the reference's edge cases: paths, stars,
    two components, isolated and dangling vertices, no edges, one vertex."""
    g = {}
    g["path"] = O.from_edges(6, [(i, i + 1) for i in range(5)] + [(i + 1, i) for i in range(5)])
    star = [(0, i) for i in range(1, 40)] + [(i, 0) for i in range(1, 40)]
    g["star"] = O.from_edges(40, star)
    two = [(0, 1), (1, 0), (1, 2), (2, 1), (3, 4), (4, 3), (4, 5), (5, 4)]
    g["two_components"] = O.from_edges(7, two)  # vertex 6 isolated
    g["dangling_directed"] = O.from_edges(5, [(0, 1), (0, 2), (1, 2), (3, 0)])  # 2, 4 have no out-edges
    g["no_edges"] = O.from_edges(4, [])
    g["one_vertex"] = O.from_edges(1, [])
    hub = [(0, i) for i in range(1, 3000)] + [(i, 0) for i in range(1, 3000)] + [(i, i + 1) for i in range(1, 2999)]
    g["hub"] = O.from_edges(3000, hub)
    return g


@pytest.fixture(scope="session")
def graphs():
    return small_graphs()
