"""New contents loaded into a resident graph (ipg_graph_refill_host), and
engines attached again to a graph of the same shape, which reuse their
device buffers: results equal the oracle's on the new contents, bit-exact
for integers and within 1e-12 for FP64 PageRank, with the same per-superstep
counts."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _relabel(g: O.CSR, seed: int) -> O.CSR:
    """The same graph with vertex ids permuted (same V and E, other rows)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(g.V).astype(np.uint64)
    row = g.row_ptr().astype(np.int64)
    deg = np.diff(row)
    src = np.repeat(np.arange(g.V, dtype=np.uint64), deg)
    ns, nd = perm[src], perm[g.adj.astype(np.uint64)]
    order = np.lexsort((nd, ns))
    ndeg = np.bincount(ns.astype(np.int64), minlength=g.V)
    idx = np.concatenate(([0], np.cumsum(ndeg)[:-1])).astype(np.uint64)
    wgt = g.wgt[order].copy() if g.wgt is not None else None
    return O.CSR(g.V, g.E, idx, nd[order].astype(np.uint32), wgt)


def _check(res, want, counts, fp=False):
    if fp:
        assert np.max(np.abs(res.values - want)) <= 1e-12
    else:
        np.testing.assert_array_equal(res.values.astype(np.uint64), want.astype(np.uint64))
    assert res.counts == [int(c) for c in counts]


def test_refill_undirected_then_rerun():
    import ipregel_b200 as ip
    a = O.add_weights(O.gen_rmat(12, 16, seed=3, undirected=True), wmax=255, seed=5)
    b = _relabel(a, seed=9)
    g = ip.Graph.from_csr(a.V, a.E, a.idx, a.adj, wgt=a.wgt)
    cc = ip.Engine("cc", "spread")
    sp = ip.Engine("sssp_weighted", "spread")
    try:
        for eng in (cc, sp):
            eng.set_quiet(True)
        sp.set_param("source", 0)
        for src in (a, b, a):
            g.refill(src.idx, src.adj, src.wgt)
            assert not g.symmetric  # the declaration belongs to the old contents
            g.set_symmetric(True)
            cc.attach(g)
            res = cc.run()
            want, counts, _ = O.run(src, "cc", "spread")
            _check(res, want, counts)
            sp.attach(g)
            res = sp.run()
            want, counts, _ = O.run(src, "sssp_weighted", "spread", source=0)
            _check(res, want, counts)
            np.testing.assert_array_equal(res.values, O.dijkstra(src, 0))
    finally:
        cc.release()
        sp.release()
        g.free()


def test_refill_directed_rebuilds_in_lists():
    import ipregel_b200 as ip
    a = O.gen_rmat(11, 8, seed=4, undirected=False)
    b = _relabel(a, seed=2)
    g = ip.Graph.from_csr(a.V, a.E, a.idx, a.adj, directed=True, need_in=True)
    try:
        for src in (b, a):
            g.refill(src.idx, src.adj)
            res = ip.run_app("pagerank", "single_broadcast", g, params={"rounds": 10})
            want, counts, _ = O.run(src, "pagerank", "single_broadcast", directed=True)
            _check(res, want, counts, fp=True)
            res = ip.run_app("cc", "single_broadcast", g)
            want, counts, _ = O.run(src, "cc", "single_broadcast", directed=True)
            _check(res, want, counts)
    finally:
        g.free()


def test_refill_rejects_bad_contents_and_sizes():
    import ipregel_b200 as ip
    a = O.gen_rmat(10, 8, seed=1, undirected=True)
    g = ip.Graph.from_csr(a.V, a.E, a.idx, a.adj)
    try:
        bad = a.adj.copy()
        bad[a.E // 2] = a.V  # an id out of range
        with pytest.raises(ip.IPregelError, match="neighbour id"):
            g.refill(a.idx, bad)
        with pytest.raises(ValueError):
            g.refill(a.idx, a.adj[:-1])
        g.refill(a.idx, a.adj)  # good contents again: usable
        res = ip.run_app("cc", "combiner", g)
        want, counts, _ = O.run(a, "cc", "combiner")
        _check(res, want, counts)
    finally:
        g.free()


def test_reattach_same_shape_and_other_shapes():
    """An engine attached in turn to graphs of the same shape (its buffers
    reused) and of other shapes (reallocated) gives each graph its own result."""
    import ipregel_b200 as ip
    a = O.gen_rmat(12, 16, seed=6, undirected=True)
    b = _relabel(a, seed=3)
    c = O.gen_rmat(10, 16, seed=7, undirected=True)
    graphs = {id(x): ip.Graph.from_csr(x.V, x.E, x.idx, x.adj) for x in (a, b, c)}
    eng = ip.Engine("sssp", "combiner")
    try:
        eng.set_quiet(True)
        eng.set_param("source", 0)
        for src in (a, b, c, a, b):
            eng.attach(graphs[id(src)])
            res = eng.run()
            want, counts, _ = O.run(src, "sssp", "combiner", source=0)
            _check(res, want, counts)
    finally:
        eng.release()
        for gr in graphs.values():
            gr.free()


def test_refill_on_a_thread_while_another_graph_runs():
    """The pipelined pattern: graph X is refilled on a second host thread
    (its own stream) while the engines run on graph Y; every step's results
    equal the oracle's for that step's contents."""
    import threading

    import ipregel_b200 as ip
    base = O.add_weights(O.gen_rmat(13, 16, seed=8, undirected=True), wmax=255, seed=2)
    contents = [base] + [_relabel(base, seed=s) for s in (1, 2, 3, 4)]
    gbuf = [ip.Graph.from_csr(base.V, base.E, base.idx, base.adj, wgt=base.wgt) for _ in range(2)]
    cc = ip.Engine("cc", "spread")
    sp = ip.Engine("sssp_weighted", "spread")
    try:
        for eng in (cc, sp):
            eng.set_quiet(True)
        sp.set_param("source", 0)
        err = []

        def refill(gr, src):
            try:
                gr.refill(src.idx, src.adj, src.wgt)
            except Exception as ex:
                err.append(ex)

        th = threading.Thread(target=refill, args=(gbuf[0], contents[0]))
        th.start()
        for k, src in enumerate(contents):
            th.join()
            assert not err, err
            if k + 1 < len(contents):
                th = threading.Thread(target=refill, args=(gbuf[(k + 1) % 2], contents[k + 1]))
                th.start()
            gr = gbuf[k % 2]
            gr.set_symmetric(True)
            cc.attach(gr)
            res = cc.run()
            want, counts, _ = O.run(src, "cc", "spread")
            _check(res, want, counts)
            sp.attach(gr)
            res = sp.run()
            np.testing.assert_array_equal(res.values, O.dijkstra(src, 0))
    finally:
        cc.release()
        sp.release()
        for gr in gbuf:
            gr.free()


def test_run_refuses_stale_attach_and_bad_contents():
    """An engine attached before a refill refuses to run until it attaches
    again (its degree classes and in-list pointers belong to the old
    contents); after a failed refill every attach and run refuses until a
    refill succeeds."""
    import ipregel_b200 as ip
    a = O.gen_rmat(11, 16, seed=12, undirected=False)
    b = _relabel(a, seed=5)
    g = ip.Graph.from_csr(a.V, a.E, a.idx, a.adj, directed=True, need_in=True)
    pr = ip.Engine("pagerank", "single_broadcast")
    cc = ip.Engine("cc", "spread")
    try:
        for eng in (pr, cc):
            eng.set_quiet(True)
            eng.attach(g)
        gen0, ok = g.contents()
        assert ok
        g.refill(b.idx, b.adj)
        gen1, ok = g.contents()
        assert ok and gen1 == gen0 + 1
        for eng in (pr, cc):
            with pytest.raises(ip.IPregelError, match="attach it again"):
                eng.run_only()
        pr.attach(g)
        res = pr.run()
        want, counts, _ = O.run(b, "pagerank", "single_broadcast", directed=True)
        _check(res, want, counts, fp=True)

        bad = b.adj.copy()
        bad[7] = b.V
        with pytest.raises(ip.IPregelError, match="neighbour id"):
            g.refill(b.idx, bad)
        assert g.contents() == (gen1 + 1, False)
        with pytest.raises(ip.IPregelError, match="failed validation"):
            pr.run_only()
        with pytest.raises(ip.IPregelError, match="failed validation"):
            cc.attach(g)
        g.refill(a.idx, a.adj)
        assert g.contents() == (gen1 + 2, True)
        cc.attach(g)
        res = cc.run()
        want, counts, _ = O.run(a, "cc", "spread", directed=True)
        _check(res, want, counts)
    finally:
        pr.release()
        cc.release()
        g.free()
