"""CUDA engine against the oracle, through the C ABI of the application
libraries (lib/app_*.so): integer applications bit-exact, FP64 PageRank
within 1e-12 max abs per vertex, and the same per-superstep
ActiveVertexCount sequence (the reference's own progress log)."""
import numpy as np
import pytest

import oracle as O
from conftest import small_graphs

pytestmark = pytest.mark.gpu

PR_TOL = 1e-12  # max abs difference per vertex, FP64 PageRank / PPR

ALL4 = ("combiner", "spread", "single_broadcast", "single_broadcast_spread")
CASES = [("cc", v) for v in ALL4] + [("sssp", v) for v in ALL4] + \
        [("pagerank", "single_broadcast"), ("pagerank", "combiner"), ("pagerank", "spread"),
         ("ppr", "single_broadcast"), ("ppr", "combiner"),
         ("sssp_weighted", "combiner"), ("sssp_weighted", "spread"),
         ("sssp_weighted_send", "combiner"), ("sssp_weighted_send", "spread")]

ORACLE_APP = {"cc": "cc", "sssp": "sssp", "pagerank": "pagerank", "ppr": "ppr",
              "sssp_weighted": "sssp_weighted", "sssp_weighted_send": "sssp_weighted"}


def _gpu_run(app, version, g, directed=False, id_bits=32, generic=False, params=None):
    import ipregel_b200 as ip
    wgt = g.wgt if app.startswith("sssp_weighted") else None
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj if id_bits == 32 else g.adj.astype(np.uint64), wgt=wgt,
                              directed=directed, id_bytes=id_bits // 8)
    try:
        return ip.run_app(app, version, graph, id_bits=id_bits, generic=generic, params=params)
    finally:
        graph.free()


def _compare(app, version, g, directed=False, id_bits=32, generic=False, source=0, rounds=None):
    params = {}
    if app in ("sssp", "sssp_weighted", "sssp_weighted_send", "ppr"):
        params["source"] = source
    if rounds is not None:
        params["rounds"] = rounds
    elif app in ("pagerank", "ppr"):
        # parameters are globals of the library: state the default explicitly
        params["rounds"] = 20 if app == "ppr" else 10
    res = _gpu_run(app, version, g, directed, id_bits, generic, params)
    kw = dict(source=source, directed=directed, id_bytes=id_bits // 8)
    if rounds is not None:
        kw["rounds"] = rounds
    elif app == "ppr":
        kw["rounds"] = 20
    want, counts, _ = O.run(g, ORACLE_APP[app], version, **kw)
    if app in ("pagerank", "ppr"):
        assert res.values.shape == want.shape
        err = np.max(np.abs(res.values - want)) if g.V else 0.0
        assert err <= PR_TOL, f"max abs error {err}"
    else:
        np.testing.assert_array_equal(res.values.astype(np.uint64), want.astype(np.uint64))
    assert res.counts == [int(c) for c in counts]
    return res


def _weighted(g):
    return O.add_weights(g, wmax=255, seed=11)


@pytest.mark.parametrize("app,version", CASES)
def test_rmat_undirected(app, version):
    g = _weighted(O.gen_rmat(12, 16, seed=1, undirected=True))
    _compare(app, version, g)


@pytest.mark.parametrize("app,version", CASES)
def test_rmat_directed_file(app, version):
    """Directed R-MAT file loaded with directed = false, as the reference's
    applications do (in-lists alias the rows)."""
    g = _weighted(O.gen_rmat(11, 16, seed=4, undirected=False))
    _compare(app, version, g)


@pytest.mark.parametrize("app,version", [("cc", "single_broadcast"), ("sssp", "single_broadcast_spread"),
                                         ("pagerank", "single_broadcast"), ("cc", "combiner")])
def test_directed_true_builds_in_lists(app, version):
    """directed = true: the pull versions gather over the true in-lists, built
    on the device in the reference's mirror order."""
    g = O.gen_rmat(10, 16, seed=9, undirected=False)
    _compare(app, version, g, directed=True)


@pytest.mark.parametrize("app,version", CASES)
def test_small_graphs(app, version):
    for name, g in small_graphs().items():
        g = _weighted(g)
        _compare(app, version, g)


@pytest.mark.parametrize("app,version", [("cc", v) for v in ALL4] + [("sssp", v) for v in ALL4])
def test_64bit_ids(app, version):
    g = O.gen_rmat(10, 16, seed=2, undirected=True)
    _compare(app, version, g, id_bits=64)


@pytest.mark.parametrize("app,version,bits", [("cc", "combiner", 32), ("cc", "spread", 32),
                                              ("pagerank", "combiner", 32), ("pagerank", "spread", 32),
                                              ("sssp", "combiner", 64), ("sssp", "spread", 64)])
def test_generic_combiner_paths(app, version, bits):
    """Builds without IP_COMBINE_KIND: delivery runs a CAS loop around the
    user's ip_combine (packed 64-bit word for 4-byte messages, 128-bit CAS for
    8-byte messages)."""
    g = O.gen_rmat(11, 16, seed=6, undirected=True)
    _compare(app, version, g, id_bits=bits, generic=True)


def test_sssp_other_sources():
    g = _weighted(O.gen_rmat(11, 16, seed=8, undirected=True))
    for src in (1, 17, 1000, 2047):
        _compare("sssp", "spread", g, source=src)
        _compare("sssp_weighted", "combiner", g, source=src)


def test_weighted_sssp_equals_dijkstra():
    g = _weighted(O.gen_rmat(12, 16, seed=12, undirected=True))
    res = _gpu_run("sssp_weighted", "spread", g, params={"source": 0})
    np.testing.assert_array_equal(res.values, O.dijkstra(g, 0))


def test_pagerank_30_rounds():
    g = O.gen_rmat(12, 16, seed=1, undirected=False)
    res = _compare("pagerank", "single_broadcast", g, rounds=30)
    assert res.supersteps == 31


def test_er_graphs():
    for n in (1024, 5000, 65536):
        g = _weighted(O.gen_er(n, 8 * n, seed=n, undirected=False))
        _compare("cc", "spread", g)
        _compare("sssp_weighted", "spread", g)


def test_send_message_in_broadcast_version_is_fatal():
    """ip_send_message under a single-broadcast version is an error, as in
    combiner_single_broadcast_postamble.h:42-49: the engine reports it."""
    import ipregel_b200 as ip
    g = _weighted(O.gen_rmat(8, 8, seed=1, undirected=True))
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
    eng = ip.Engine("sssp_weighted_send", "single_broadcast")
    eng.set_quiet()
    eng.attach(graph)
    with pytest.raises(ip.IPregelError, match="send_message should not be used"):
        eng.run()
    # the context stays usable: the same process runs another engine afterwards
    eng.release()
    res = ip.run_app("cc", "combiner", graph)
    want, _, _ = O.run(g, "cc", "combiner")
    np.testing.assert_array_equal(res.values, want)
    graph.free()


PULL_CASES = [("cc", "combiner"), ("cc", "spread"), ("sssp", "combiner"), ("sssp", "spread"),
              ("sssp_weighted", "combiner"), ("sssp_weighted", "spread"), ("sssp_weighted_send", "spread"),
              ("pagerank", "combiner"), ("pagerank", "spread"), ("ppr", "combiner")]


@pytest.mark.parametrize("app,version", PULL_CASES)
@pytest.mark.parametrize("div", ["1000000000", "3"])
def test_pull_delivery_on_symmetric_graphs(app, version, div, monkeypatch):
    """Push versions on a graph declared symmetric deliver dense supersteps by
    pulling over the rows (always, with a huge IPG_PULL_DIV, or past E/3):
    same results as the oracle's push."""
    import ipregel_b200 as ip
    monkeypatch.setenv("IPG_PULL_DIV", div)
    g = _weighted(O.gen_rmat(12, 16, seed=13, undirected=True))
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
    assert graph.check_symmetric() == 1
    graph.set_symmetric(True)
    params = {"source": 0} if app in ("sssp", "sssp_weighted", "sssp_weighted_send", "ppr") else {}
    try:
        res = ip.run_app(app, version, graph, params=params)
    finally:
        graph.free()
    kw = {"rounds": 20} if app == "ppr" else {}
    want, counts, _ = O.run(g, ORACLE_APP[app], version, **kw)
    if app in ("pagerank", "ppr"):
        assert np.max(np.abs(res.values - want)) <= PR_TOL
    else:
        np.testing.assert_array_equal(res.values, want)
    assert res.counts == [int(c) for c in counts]


def test_symmetry_check_and_generator_flag():
    import ipregel_b200 as ip
    und = ip.Graph.generate_rmat(10, 8, seed=2, undirected=True, wmax=9)
    assert und.symmetric and und.check_symmetric() == 1
    d = ip.Graph.generate_rmat(10, 8, seed=2, undirected=False)
    assert not d.symmetric and d.check_symmetric() == 0
    g = O.from_edges(3, [(0, 2), (0, 1), (1, 0), (2, 0)])  # row 0 not sorted
    u = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    assert u.check_symmetric() == -1
    for x in (und, d, u):
        x.free()


@pytest.mark.parametrize("app", ["pagerank", "cc", "sssp"])
@pytest.mark.parametrize("t0,t1", [(16, 4096), (2, 64), (1, 1), (64, 100000)])
@pytest.mark.parametrize("hot_kb", ["0", "4", "65536"])
def test_single_broadcast_degree_classes(app, t0, t1, hot_kb, monkeypatch):
    """The single_broadcast gather fused with the next superstep's compute,
    over every split of the in-degree classes: hubs in many chunks of 2048
    in-edges folded by whichever CTA arrives last (t1 = 1, 64), hubs in one
    chunk, rows of every alignment read 128 bits at a time by warps and
    blocks; with none, some or all in-neighbours flagged for the L2
    (IPG_SB_HOT_KB); host and captured loops; per-superstep counts
    identical."""
    import ipregel_b200 as ip
    monkeypatch.setenv("IPG_SB_HOT_KB", hot_kb)
    hub = [(0, i) for i in range(1, 9000)] + [(i, 0) for i in range(1, 9000)] + \
          [(i, i + 1) for i in range(1, 8999)] + [(i + 1, i) for i in range(1, 8999)] + [(5, 7000), (7000, 5)]
    graphs = [O.gen_rmat(12, 16, seed=21, undirected=False), O.from_edges(9000, hub),
              O.gen_rmat(11, 16, seed=22, undirected=True)]
    for g in graphs:
        graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
        eng = ip.Engine(app, "single_broadcast")
        try:
            eng.set_quiet(True)
            eng.set_tuning(t0=t0, t1=t1)
            params = {"rounds": 10} if app == "pagerank" else {"source": 3} if app == "sssp" else {}
            for k, v in params.items():
                eng.set_param(k, v)
            want, counts, _ = O.run(g, app, "single_broadcast", source=params.get("source", 0))
            for loop in (False, True):
                eng.set_graph_loop(loop)
                eng.attach(graph)
                for _ in range(2):  # a second run on the same attachment
                    res = eng.run()
                    if app == "pagerank":
                        assert np.max(np.abs(res.values - want)) <= PR_TOL
                    else:
                        np.testing.assert_array_equal(res.values, want)
                    assert res.counts == [int(c) for c in counts]
        finally:
            eng.release()
            graph.free()


@pytest.mark.parametrize("app", ["pagerank", "cc"])
def test_single_broadcast_staged_hub_chunks(app):
    """The build whose pull gather takes a CTA per hub chunk with the chunk's
    ids staged in shared memory by bulk copies (appstaged_*): the same
    results as the oracle, with many chunks per hub (t1 = 64) and one."""
    import ipregel_b200 as ip
    hub = [(0, i) for i in range(1, 9000)] + [(i, 0) for i in range(1, 9000)] + \
          [(i, i + 1) for i in range(1, 8999)] + [(i + 1, i) for i in range(1, 8999)]
    for g in (O.gen_rmat(12, 16, seed=31, undirected=False), O.from_edges(9000, hub)):
        graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
        eng = ip.Engine(app, "single_broadcast", variant="staged")
        try:
            eng.set_quiet(True)
            if app == "pagerank":
                eng.set_param("rounds", 10)
            want, counts, _ = O.run(g, app, "single_broadcast")
            for t1 in (64, 4096):
                eng.set_tuning(t0=16, t1=t1)
                for loop in (False, True):
                    eng.set_graph_loop(loop)
                    eng.attach(graph)
                    res = eng.run()
                    if app == "pagerank":
                        assert np.max(np.abs(res.values - want)) <= PR_TOL
                    else:
                        np.testing.assert_array_equal(res.values, want)
                    assert res.counts == [int(c) for c in counts]
        finally:
            eng.release()
            graph.free()


def test_reserved_fp64_pattern_is_refused():
    """The single_broadcast engine's 8-byte FP64 slots keep the all-ones bit
    pattern for "no broadcast": a program that broadcasts exactly that
    pattern gets an error (host and captured loops), a program that does not
    gets its results, and the engine stays usable after the error."""
    import ipregel_b200 as ip
    g = O.gen_rmat(9, 8, seed=3, undirected=True)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    eng = ip.Engine("reserved", "single_broadcast")
    try:
        eng.set_quiet(True)
        src = int(np.argmax(np.diff(g.row_ptr())))  # a vertex with edges
        eng.set_param("source", src)
        row = g.row_ptr().astype(np.int64)
        want = np.array([float(np.count_nonzero(g.adj[row[v]:row[v + 1]] == src)) for v in range(g.V)])
        for loop in (False, True):
            eng.set_graph_loop(loop)
            eng.attach(graph)
            eng.set_param("allones", 0)
            res = eng.run()
            np.testing.assert_array_equal(res.values, want)
            eng.set_param("allones", 1)
            with pytest.raises(ip.IPregelError, match="all 64 bits set"):
                eng.run()
            eng.set_param("allones", 0)
            np.testing.assert_array_equal(eng.run().values, want)
    finally:
        eng.set_graph_loop(False)
        eng.release()
        graph.free()
