"""PageRank precision split (ipg_pr_run_f32): FP32 values with compensated
gather sums against the FP64 oracle (the reference's pagerank.c formula under
the single-broadcast version), FP64 diagnostics against sums taken over the
oracle's values, and the error-report kernel.

Tolerance: max relative error per vertex <= 1e-5 against FP64 (each superstep
adds a few FP32 roundings, about 3 * 2^-24 relative, which the damping 0.85
contracts: the fixed point is off by at most 3 * 2^-24 / 0.15, about 1.2e-6)."""
import numpy as np
import pytest

import oracle as O
from conftest import small_graphs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


def _rel_err(x, want):
    den = np.where(want != 0, np.abs(want), 1.0)
    return np.max(np.abs(x.astype(np.float64) - want) / den) if want.size else 0.0


def _run(g, rounds, compensated=True, damping=0.85):
    import ipregel_b200 as ip
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    pr = ip.PageRankF32(graph)
    try:
        return pr.run(rounds=rounds, damping=damping, compensated=compensated) + (pr.info(),)
    finally:
        pr.free()
        graph.free()


@pytest.mark.parametrize("rounds", [10, 30])
def test_rmat16_directed_against_fp64_oracle(rounds):
    """The small PageRank workload: directed R-MAT scale 16, edge factor 16,
    seed 1, 10 rounds (pagerank.c as shipped) and 30."""
    g = O.gen_rmat(16, 16, seed=1, undirected=False)
    x, diag, info = _run(g, rounds)
    want, counts, _ = O.run(g, "pagerank", "single_broadcast", rounds=rounds)
    assert len(counts) == rounds + 1
    assert _rel_err(x, want) <= REL_TOL
    assert diag.shape == (rounds + 1, 3)
    # FP64 diagnostics of the last superstep against sums over the oracle's values
    deg = np.diff(g.idx.astype(np.int64), append=g.E)
    assert diag[-1, 0] == pytest.approx(want.sum(), rel=REL_TOL)
    assert diag[-1, 1] == pytest.approx(want[deg == 0].sum(), rel=REL_TOL, abs=1e-12)
    prev, _, _ = O.run(g, "pagerank", "single_broadcast", rounds=rounds - 1)
    assert diag[-1, 2] == pytest.approx(np.abs(want - prev).sum(), rel=1e-3, abs=1e-9)
    assert diag[0, 0] == pytest.approx(1.0, rel=1e-6) and diag[0, 2] == 0.0


def test_undirected_hubs_split_into_chunks():
    """Undirected R-MAT scale 15: hubs above 4096 edges take the chunked path."""
    g = O.gen_rmat(15, 16, seed=2, undirected=True)
    x, diag, info = _run(g, 20)
    assert info["class_counts"][2] > 0 and info["hub_chunks"] > info["class_counts"][2]
    want, _, _ = O.run(g, "pagerank", "single_broadcast", rounds=20)
    assert _rel_err(x, want) <= REL_TOL


def test_compensation_reduces_error():
    g = O.gen_rmat(15, 16, seed=3, undirected=True)
    want, _, _ = O.run(g, "pagerank", "single_broadcast", rounds=30)
    xc, _, _ = _run(g, 30, compensated=True)
    xp, _, _ = _run(g, 30, compensated=False)
    ec, ep = _rel_err(xc, want), _rel_err(xp, want)
    assert ec <= REL_TOL
    assert ec <= ep


def test_deterministic_values():
    g = O.gen_rmat(14, 16, seed=4, undirected=True)
    a, _, _ = _run(g, 10)
    b, _, _ = _run(g, 10)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


def test_small_graphs_and_rounds_zero():
    for name, g in small_graphs().items():
        for rounds in (0, 1, 5):
            x, diag, _ = _run(g, rounds)
            assert x.shape == (g.V,), name
            if g.V == 0:
                continue
            want, _, _ = O.run(g, "pagerank", "single_broadcast", rounds=rounds)
            assert _rel_err(x, want) <= REL_TOL, (name, rounds)


def test_damping_parameter():
    g = O.gen_rmat(12, 8, seed=5, undirected=False)
    x, _, _ = _run(g, 10, damping=0.5)
    # restated FP64 iteration with damping 0.5
    V = g.V
    deg = np.diff(g.idx.astype(np.int64), append=g.E)
    src = np.repeat(np.arange(V), deg)
    xv = np.full(V, 1.0 / V)
    for _ in range(10):
        q = np.where(deg > 0, xv / np.maximum(deg, 1), 0.0)
        s = np.zeros(V)
        np.add.at(s, src, q[g.adj.astype(np.int64)])
        xv = 0.5 / V + 0.5 * s
    assert _rel_err(x, xv) <= REL_TOL


def test_error_report_kernel():
    import ipregel_b200 as ip
    ref = np.array([1.0, 2.0, 0.0, 4.0, -8.0])
    a = np.array([1.0, 2.5, 0.25, 4.0, -8.5], dtype=np.float32)
    da, dr = ip.DeviceArray(5, np.float32), ip.DeviceArray(5, np.float64)
    try:
        da.from_host(a)
        dr.from_host(ref)
        e = ip.error_f32_f64(da, dr)
    finally:
        da.free()
        dr.free()
    assert e["max_abs"] == 0.5 and e["argmax_abs"] == 1
    assert e["max_rel"] == 0.25 and e["mean_abs"] == pytest.approx(1.25 / 5)


def test_directed_flag_selects_gather_lists():
    """directed = false gathers over the rows (the reference's benchmarks);
    directed = true over the transpose, as the FP64 engine does."""
    import ipregel_b200 as ip
    g = O.gen_rmat(13, 16, seed=6, undirected=False)
    graph = ip.Graph.generate_rmat(13, 16, seed=6, undirected=False)
    try:
        assert graph.V == g.V and graph.E == g.E
        for directed in (True, False, True):
            graph.set_directed(directed)
            pr = ip.PageRankF32(graph)
            x, _ = pr.run(rounds=15)
            pr.free()
            want, _, _ = O.run(g, "pagerank", "single_broadcast", rounds=15, directed=directed)
            assert _rel_err(x, want) <= REL_TOL, directed
            res = ip.run_app("pagerank", "single_broadcast", graph, params={"rounds": 15})
            assert np.max(np.abs(res.values - want)) <= 1e-12
    finally:
        # application parameters are globals of the library: restore the default
        ip.Engine("pagerank", "single_broadcast").set_param("rounds", 10)
        graph.free()


def test_64bit_ids_rejected():
    import ipregel_b200 as ip
    g = O.gen_rmat(8, 8, seed=1, undirected=False)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj.astype(np.uint64), id_bytes=8)
    try:
        with pytest.raises(ip.IPregelError, match="32-bit"):
            ip.PageRankF32(graph)
    finally:
        graph.free()
