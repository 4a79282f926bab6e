"""ipg_degree_classes_noalloc -- the entry point for callers that cannot
allocate device memory (stream capture in progress, latency-bound serving
loops, host programs whose pool owns all of HBM).  Called through the C ABI
and compared, call after call, with ipg_graph_bins, which computes the same
degree classes with its own temporary allocations.  The file sorts last so
that a run stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_V = 67108864


def _cudart():
    lib = ctypes.CDLL("libcudart.so.12")
    lib.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    lib.cudaMemset.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t]
    lib.cudaDeviceSynchronize.argtypes = []
    return lib


def _d2h(rt, dptr, n, dtype):
    out = np.zeros(max(n, 1), dtype=dtype)
    if n:
        assert rt.cudaMemcpy(out.ctypes.data, dptr, n * out.itemsize, 2) == 0
    return out[:n]


def _alloc(lib, nbytes):
    p = ctypes.c_void_p()
    assert lib.ipg_dev_alloc(ctypes.byref(p), nbytes) == 0
    return p


def _reference_bins(lib, rt, graph, t0, t1):
    import ipregel_b200 as ip

    class Bins(ctypes.Structure):
        _fields_ = [("d_list", ctypes.c_void_p * 3), ("count", ctypes.c_uint64 * 3),
                    ("edges", ctypes.c_uint64 * 3), ("t0", ctypes.c_uint64), ("t1", ctypes.c_uint64)]

    b = Bins()
    lib.ipg_graph_bins.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                   ctypes.POINTER(Bins)]
    assert lib.ipg_graph_bins(graph.handle, 0, t0, t1, ctypes.byref(b)) == 0, ip.runtime().ipg_last_error()
    counts = [int(c) for c in b.count]
    lists = np.concatenate([_d2h(rt, b.d_list[k], counts[k], np.uint32) for k in range(3)])
    return lists, counts, [int(e) for e in b.edges]


@pytest.mark.parametrize("t0,t1", [(16, 4096), (0, 32), (3, 3)])
def test_noalloc_matches_allocating_entry_point(t0, t1):
    import ipregel_b200 as ip
    lib = ip.runtime()
    rt = _cudart()
    fn = lib.ipg_degree_classes_noalloc
    fn.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    graphs = [ip.Graph.generate_rmat(16, 16, seed=3, undirected=True),
              ip.Graph.generate_rmat(13, 8, seed=4, undirected=False),
              ip.Graph.generate_er(70001, 8 * 70001, seed=5)]
    try:
        for g in graphs:
            V = g.V
            want_lists, want_counts, want_edges = _reference_bins(lib, rt, g, t0, t1)
            d_lists = _alloc(lib, V * 4)
            d_totals = _alloc(lib, 6 * 8)
            try:
                for call in range(2):
                    # poison the outputs so that every element must be written again
                    assert rt.cudaMemset(d_lists, 0xAB, V * 4) == 0
                    assert rt.cudaMemset(d_totals, 0xCD, 48) == 0
                    held = ip.hbm_in_use()
                    rc = fn(V, g.view.d_row, t0, t1, d_lists, d_totals, None)
                    assert rc == 0, lib.ipg_last_error()
                    assert rt.cudaDeviceSynchronize() == 0
                    assert ip.hbm_in_use() == held  # nothing allocated through the library
                    totals = _d2h(rt, d_totals, 6, np.uint64)
                    assert [int(x) for x in totals[:3]] == want_counts, (call, V)
                    assert [int(x) for x in totals[3:]] == want_edges, (call, V)
                    np.testing.assert_array_equal(_d2h(rt, d_lists, V, np.uint32), want_lists)
            finally:
                lib.ipg_dev_free(d_lists, V * 4)
                lib.ipg_dev_free(d_totals, 48)
    finally:
        for g in graphs:
            g.free()


def test_noalloc_rejects_graphs_above_the_limit():
    import ipregel_b200 as ip
    lib = ip.runtime()
    fn = lib.ipg_degree_classes_noalloc
    fn.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    assert fn(MAX_V + 1, dummy, 16, 4096, dummy, dummy, None) == -1
    assert b"at most 67108864 vertices" in lib.ipg_last_error()
