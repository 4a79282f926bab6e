"""The degree-ordered copy the engine runs on (ipg_graph_degree_order): the
copy is a renaming of the graph that keeps every row's edge order, and every
application gives the same values and per-superstep counts on it as on the
graph's own numbering, both equal to the oracle's."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import small_graphs

pytestmark = pytest.mark.gpu

ORDER_DEFAULT = os.environ.get("IPG_ORDER", "1") != "0"

ALL4 = ("combiner", "spread", "single_broadcast", "single_broadcast_spread")
CASES = [("cc", v) for v in ALL4] + [("sssp", v) for v in ALL4] + \
        [("pagerank", "single_broadcast"), ("pagerank", "combiner"), ("pagerank", "spread"),
         ("ppr", "single_broadcast"), ("ppr", "combiner"),
         ("sssp_weighted", "combiner"), ("sssp_weighted", "spread"),
         ("sssp_weighted_send", "combiner"), ("sssp_weighted_send", "spread")]
ORACLE_APP = {"cc": "cc", "sssp": "sssp", "pagerank": "pagerank", "ppr": "ppr", "sssp_weighted": "sssp_weighted",
              "sssp_weighted_send": "sssp_weighted"}
PR_TOL = 1e-12


def _params(app):
    p = {}
    if app in ("sssp", "sssp_weighted", "sssp_weighted_send", "ppr"):
        p["source"] = 0
    if app in ("pagerank", "ppr"):
        p["rounds"] = 20 if app == "ppr" else 10
    return p


def _run(app, version, graph, order, params=None, id_bits=32):
    import ipregel_b200 as ip
    eng = ip.Engine(app, version, id_bits)
    eng.set_quiet(True)
    try:
        eng.set_order(order)
        for k, v in (params if params is not None else _params(app)).items():
            eng.set_param(k, v)
        eng.attach(graph)
        assert eng.order() == order
        return eng.run()
    finally:
        eng.set_order(ORDER_DEFAULT)


def _both(app, version, g, directed=False, id_bits=32):
    import ipregel_b200 as ip
    wgt = g.wgt if app.startswith("sssp_weighted") else None
    adj = g.adj if id_bits == 32 else g.adj.astype(np.uint64)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, adj, wgt=wgt, directed=directed, id_bytes=id_bits // 8)
    try:
        off = _run(app, version, graph, False, id_bits=id_bits)
        on = _run(app, version, graph, True, id_bits=id_bits)
    finally:
        graph.free()
    assert on.counts == off.counts
    kw = dict(source=0, directed=directed, id_bytes=id_bits // 8)
    if app == "ppr":
        kw["rounds"] = 20
    want, counts, _ = O.run(g, ORACLE_APP[app], version, **kw)
    assert on.counts == [int(c) for c in counts]
    if app in ("pagerank", "ppr"):
        # FP64 sums: the warp classes' 128-bit loads split a row by its
        # offset modulo 4, which the renaming moves, so the two runs may
        # differ in the last bits (the thread class folds in row order in both)
        assert np.max(np.abs(on.values - want)) <= PR_TOL
        assert np.max(np.abs(on.values - off.values)) <= PR_TOL
    else:
        np.testing.assert_array_equal(on.values, off.values)
        np.testing.assert_array_equal(on.values.astype(np.uint64), want.astype(np.uint64))


@pytest.mark.parametrize("app,version", CASES)
def test_renamed_equals_own_numbering_rmat(app, version):
    _both(app, version, O.add_weights(O.gen_rmat(12, 16, seed=3, undirected=True), wmax=255, seed=5))


@pytest.mark.parametrize("app,version", CASES)
def test_renamed_equals_own_numbering_directed_file(app, version):
    _both(app, version, O.add_weights(O.gen_rmat(11, 16, seed=6, undirected=False), wmax=255, seed=7))


@pytest.mark.parametrize("app,version", [("cc", "single_broadcast"), ("sssp", "single_broadcast_spread"),
                                         ("pagerank", "single_broadcast"), ("cc", "combiner")])
def test_renamed_in_lists_of_directed_graph(app, version):
    """directed = true: the in-lists are the transpose, renamed from the
    graph's own (so each keeps the reference's source order)."""
    _both(app, version, O.gen_rmat(10, 8, seed=9, undirected=False), directed=True)


@pytest.mark.parametrize("app,version", [("cc", "spread"), ("sssp", "combiner"), ("cc", "single_broadcast")])
def test_renamed_64bit_ids(app, version):
    _both(app, version, O.gen_rmat(10, 16, seed=2, undirected=True), id_bits=64)


@pytest.mark.parametrize("app,version", [("cc", "combiner"), ("sssp", "spread"), ("pagerank", "single_broadcast")])
def test_renamed_small_graphs(app, version):
    for name, g in small_graphs().items():
        _both(app, version, g)


def test_degree_order_is_a_renaming():
    import ipregel_b200 as ip
    g = O.add_weights(O.gen_rmat(10, 8, seed=12, undirected=False), wmax=1000, seed=1)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt, directed=True)
    try:
        c = graph.degree_order(need_in=True)
    finally:
        graph.free()
    V, E = g.V, g.E
    o2n, n2o = c["old_of_new"].astype(np.int64), c["new_of_old"].astype(np.int64)
    np.testing.assert_array_equal(np.sort(o2n), np.arange(V))
    np.testing.assert_array_equal(n2o[o2n], np.arange(V))
    occ = np.bincount(g.adj.astype(np.int64), minlength=V)
    k = occ[o2n]
    assert np.all(k[:-1] >= k[1:])  # descending occurrences
    ties = k[:-1] == k[1:]
    assert np.all(o2n[:-1][ties] < o2n[1:][ties])  # ties by ascending id
    row = np.append(g.idx.astype(np.int64), E)
    nrow = c["row"].astype(np.int64)
    for n in range(V):
        o = o2n[n]
        a, b = row[o], row[o + 1]
        assert nrow[n + 1] - nrow[n] == b - a
        np.testing.assert_array_equal(c["adj"][nrow[n]:nrow[n + 1]], n2o[g.adj[a:b]])
        np.testing.assert_array_equal(c["wgt"][nrow[n]:nrow[n + 1]], g.wgt[a:b])
    # in-lists: the graph's own transpose (sources ascending), renamed
    assert c["has_in"] and not c["in_alias"]
    src = np.repeat(np.arange(V), np.diff(row))
    irow = c["in_row"].astype(np.int64)
    for n in range(V):
        o = o2n[n]
        own = src[g.adj == o]  # in-neighbours of o, ascending
        np.testing.assert_array_equal(c["in_adj"][irow[n]:irow[n + 1]], n2o[own])


def test_refill_rebuilds_the_renamed_copy():
    """A refill of the same shape rebuilds the copy in place: the next
    attach runs on the new contents."""
    import ipregel_b200 as ip
    a = O.gen_rmat(11, 16, seed=21, undirected=True)
    perm = np.random.default_rng(3).permutation(a.V).astype(np.uint32)
    b = O.CSR(a.V, a.E, a.idx.copy(), perm[a.adj])  # the same shape, other edges
    graph = ip.Graph.from_csr(a.V, a.E, a.idx, a.adj)
    try:
        first = _run("cc", "spread", graph, True)
        want_a, _, _ = O.run(a, "cc", "spread")
        np.testing.assert_array_equal(first.values.astype(np.uint64), want_a.astype(np.uint64))
        graph.refill(b.idx, b.adj)
        second = _run("cc", "spread", graph, True)
        want_b, counts_b, _ = O.run(b, "cc", "spread")
        np.testing.assert_array_equal(second.values.astype(np.uint64), want_b.astype(np.uint64))
        assert second.counts == [int(c) for c in counts_b]
    finally:
        graph.free()


@pytest.mark.parametrize("version", ["combiner", "spread"])
@pytest.mark.parametrize("mul,add", [(1, 1), (3, 7), (2, 0)])
def test_send_message_to_ids_when_renamed(version, mul, add):
    """ip_send_message names vertices by the caller's ids, renamed or not."""
    import ipregel_b200 as ip
    g = O.gen_rmat(10, 16, seed=5, undirected=True)
    V = g.V
    ids = np.arange(V, dtype=np.uint64)
    to = (ids * mul + add) % V
    want = np.full(V, 0xFFFFFFFF, dtype=np.uint64)
    np.minimum.at(want, to, ids)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    try:
        for order in (False, True):
            res = _run("ring", version, graph, order, params={"mul": mul, "add": add})
            np.testing.assert_array_equal(res.values.astype(np.uint64), want)
    finally:
        graph.free()


def test_degree_order_of_a_symmetric_graph():
    """Declared symmetric: the occurrences are the row lengths (no count pass)."""
    import ipregel_b200 as ip
    g = O.gen_rmat(10, 8, seed=13, undirected=True)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    try:
        graph.set_symmetric(True)
        c = graph.degree_order()
    finally:
        graph.free()
    o2n = c["old_of_new"].astype(np.int64)
    occ = np.bincount(g.adj.astype(np.int64), minlength=g.V)
    np.testing.assert_array_equal(occ, np.diff(np.append(g.idx.astype(np.int64), g.E)))  # symmetric rows
    k = occ[o2n]
    assert np.all(k[:-1] >= k[1:])
    ties = k[:-1] == k[1:]
    assert np.all(o2n[:-1][ties] < o2n[1:][ties])
    assert c["in_alias"] or not c["has_in"]


@pytest.mark.parametrize("undirected,directed", [(True, False), (False, True)])
def test_copy_gains_in_lists_in_place(undirected, directed):
    """A push program attached first (no in-lists), then a pull program on
    the same graph: the copy gains in-lists without moving what the first
    engine runs on, which still gives the oracle's labels."""
    import ipregel_b200 as ip
    g = O.gen_rmat(11, 16, seed=17, undirected=undirected)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, directed=directed)
    cc = ip.Engine("cc", "combiner")
    pr = ip.Engine("pagerank", "single_broadcast")
    try:
        for e in (cc, pr):
            e.set_quiet(True)
            e.set_order(True)
        pr.set_param("rounds", 10)
        cc.attach(graph)
        first = cc.run()
        pr.attach(graph)
        res_pr = pr.run()
        again = cc.run()
        want_cc, counts, _ = O.run(g, "cc", "combiner", directed=directed)
        np.testing.assert_array_equal(again.values.astype(np.uint64), want_cc.astype(np.uint64))
        np.testing.assert_array_equal(first.values, again.values)
        assert again.counts == [int(c) for c in counts]
        want_pr, _, _ = O.run(g, "pagerank", "single_broadcast", rounds=10, directed=directed)
        assert np.max(np.abs(res_pr.values - want_pr)) <= PR_TOL
    finally:
        for e in (cc, pr):
            e.set_order(ORDER_DEFAULT)
        graph.free()


def test_set_directed_makes_attached_engines_attach_again():
    import ipregel_b200 as ip
    g = O.gen_rmat(10, 16, seed=18, undirected=False)
    graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, directed=False)
    try:
        eng = ip.Engine("cc", "spread")
        eng.set_quiet(True)
        eng.attach(graph)
        eng.run()
        graph.set_directed(True)
        with pytest.raises(ip.IPregelError):
            eng.run()
        eng.attach(graph)
        res = eng.run()
        want, _, _ = O.run(g, "cc", "spread", directed=True)
        np.testing.assert_array_equal(res.values.astype(np.uint64), want.astype(np.uint64))
    finally:
        graph.free()
