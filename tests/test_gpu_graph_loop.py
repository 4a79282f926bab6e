"""The captured superstep loop (one CUDA graph with a device-evaluated while
condition per ip_run) against the oracle: same values and the same
per-superstep ActiveVertexCount sequence as the host-driven loop, repeated
runs through the cached graph, the superstep bound and error reporting from
inside the graph."""
import numpy as np
import pytest

import oracle as O
from conftest import small_graphs

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12

ALL4 = ("combiner", "spread", "single_broadcast", "single_broadcast_spread")
CASES = [("cc", v) for v in ALL4] + [("sssp", v) for v in ALL4] + \
        [("pagerank", "single_broadcast"), ("pagerank", "combiner"), ("pagerank", "spread"),
         ("ppr", "combiner"), ("sssp_weighted", "combiner"), ("sssp_weighted", "spread")]
SOURCED = ("sssp", "sssp_weighted", "sssp_weighted_send", "ppr")
ORACLE_APP = {"cc": "cc", "sssp": "sssp", "pagerank": "pagerank", "ppr": "ppr",
              "sssp_weighted": "sssp_weighted", "sssp_weighted_send": "sssp_weighted"}


def _engine(app, version):
    import ipregel_b200 as ip
    eng = ip.Engine(app, version)
    eng.set_quiet(True)
    if app in SOURCED:
        eng.set_param("source", 0)
    if app in ("pagerank", "ppr"):
        # parameters are globals of the library: state the default explicitly
        eng.set_param("rounds", 20 if app == "ppr" else 10)
    return eng


def _check(app, version, g, res):
    kw = {"rounds": 20} if app == "ppr" else {}
    want, counts, _ = O.run(g, ORACLE_APP[app], version, **kw)
    if app in ("pagerank", "ppr"):
        err = np.max(np.abs(res.values - want)) if g.V else 0.0
        assert err <= PR_TOL, f"max abs error {err}"
    else:
        np.testing.assert_array_equal(res.values, want)
    assert res.counts == [int(c) for c in counts]


@pytest.mark.parametrize("app,version", CASES)
def test_graph_loop_matches_oracle(app, version):
    import ipregel_b200 as ip
    g = O.add_weights(O.gen_rmat(12, 16, seed=3, undirected=True), wmax=255, seed=11)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
    eng = _engine(app, version)
    eng.set_graph_loop(True)
    try:
        eng.attach(graph)
        l0 = eng.launches()
        first = eng.run()
        _check(app, version, g, first)
        l1 = eng.launches()
        second = eng.run()  # the cached graph, state reset in between
        _check(app, version, g, second)
        assert eng.launches() - l1 == l1 - l0 > 0
    finally:
        eng.set_graph_loop(False)
        eng.release()
        graph.free()


@pytest.mark.parametrize("app,version", [("cc", v) for v in ALL4] + [("sssp_weighted", "spread")])
def test_graph_loop_small_graphs(app, version):
    import ipregel_b200 as ip
    eng = _engine(app, version)
    eng.set_graph_loop(True)
    try:
        for name, g in small_graphs().items():
            g = O.add_weights(g, wmax=255, seed=11)
            graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
            try:
                eng.attach(graph)
                _check(app, version, g, eng.run())
            finally:
                eng.release()
                graph.free()
    finally:
        eng.set_graph_loop(False)


@pytest.mark.parametrize("app,version", [("cc", "combiner"), ("sssp_weighted", "spread")])
def test_graph_loop_with_pull_delivery(app, version, monkeypatch):
    """Direction decided on the device inside the captured body."""
    import ipregel_b200 as ip
    monkeypatch.setenv("IPG_PULL_DIV", "3")
    g = O.add_weights(O.gen_rmat(12, 16, seed=13, undirected=True), wmax=255, seed=11)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
    graph.set_symmetric(True)
    eng = _engine(app, version)
    eng.set_graph_loop(True)
    try:
        eng.attach(graph)
        _check(app, version, g, eng.run())
    finally:
        eng.set_graph_loop(False)
        eng.release()
        graph.free()


@pytest.mark.parametrize("mode", [False, True])
def test_superstep_limit(mode, monkeypatch):
    """IPG_MAX_SUPERSTEPS bounds a run in both loops: a path of 40 vertices
    needs 40 supersteps of SSSP; a bound of 8 reports an error and leaves the
    context usable."""
    import ipregel_b200 as ip
    monkeypatch.setenv("IPG_MAX_SUPERSTEPS", "8")
    n = 40
    edges = [(i, i + 1) for i in range(n - 1)] + [(i + 1, i) for i in range(n - 1)]
    g = O.from_edges(n, edges)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    eng = _engine("sssp", "spread")
    eng.set_graph_loop(mode)
    try:
        eng.attach(graph)
        with pytest.raises(ip.IPregelError, match="superstep limit"):
            eng.run_only()
        monkeypatch.setenv("IPG_MAX_SUPERSTEPS", "1000")
        eng.release()
        eng.attach(graph)
        _check("sssp", "spread", g, eng.run())
    finally:
        eng.set_graph_loop(False)
        eng.release()
        graph.free()


def test_send_in_broadcast_version_inside_graph():
    import ipregel_b200 as ip
    g = O.add_weights(O.gen_rmat(8, 8, seed=1, undirected=True), wmax=255, seed=11)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
    eng = _engine("sssp_weighted_send", "single_broadcast")
    eng.set_graph_loop(True)
    try:
        eng.attach(graph)
        with pytest.raises(ip.IPregelError, match="send_message should not be used"):
            eng.run_only()
    finally:
        eng.set_graph_loop(False)
        eng.release()
        graph.free()
