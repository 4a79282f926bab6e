"""Request server: every served query equals the oracle (SSSP and CC exactly,
PPR within 2e-6 max abs against the FP64 ppr program), a query's result is
bitwise the same alone and in a mix, queries joining while others run
(continuous batching) stay correct, and a tight HBM budget still serves
everything by evicting idle lane groups."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

PPR_TOL = 2e-6  # FP32 lanes against the FP64 oracle, max abs per vertex


def _graphs():
    gs = [O.add_weights(O.gen_rmat(10, 8, seed=1, undirected=True), wmax=255, seed=1),
          O.add_weights(O.gen_er(3000, 12000, seed=2, undirected=True), wmax=255, seed=2),
          O.add_weights(O.gen_rmat(12, 16, seed=3, undirected=True), wmax=255, seed=3)]
    return gs


def _device(gs):
    import ipregel_b200 as ip
    return [ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt) for g in gs]


def _want(g, kind, src):
    from ipregel_b200 import serve as S
    if kind == S.SSSP:
        return O.dijkstra(g, src)
    if kind == S.CC:
        return O.run(g, "cc", "spread")[0]
    return O.run(g, "ppr", "single_broadcast", source=src, rounds=20)[0]


def _check(g, kind, src, got):
    from ipregel_b200 import serve as S
    want = _want(g, kind, src)
    if kind == S.PPR:
        assert np.max(np.abs(got.astype(np.float64) - want)) <= PPR_TOL
    else:
        np.testing.assert_array_equal(got, want)


def _queries(gs, n, seed):
    from ipregel_b200 import serve as S
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        gid = int(rng.integers(len(gs)))
        kind = int(rng.choice([S.SSSP, S.PPR, S.CC], p=[0.6, 0.3, 0.1]))
        src = 0 if kind == S.CC else int(rng.integers(gs[gid].V))
        out.append((gid, kind, src))
    return out


def test_mixed_batch_matches_oracle_and_alone():
    from ipregel_b200 import serve as S
    gs = _graphs()
    dg = _device(gs)
    srv = S.Server(ppr_rounds=20)
    try:
        for d in dg:
            srv.add_graph(d)
        qs = _queries(gs, 60, seed=1)
        ids = [srv.submit(*q) for q in qs]
        srv.drain()
        mix = []
        for qid, (gid, kind, src) in zip(ids, qs):
            assert srv.query(qid)["state"] == S.DONE
            r = srv.result(qid, kind, gs[gid].V)
            _check(gs[gid], kind, src, r)
            mix.append(r)
            srv.release(qid)
        st = srv.stats()
        assert st["submitted"] == 60 and st["lanes_admitted"] <= 60
        # alone: bitwise the same
        for (gid, kind, src), r in list(zip(qs, mix))[:12]:
            alone, _ = S.run_alone(srv, gid, kind, src, gs[gid].V)
            np.testing.assert_array_equal(alone.view(np.uint32), r.view(np.uint32))
    finally:
        srv.free()
        for d in dg:
            d.free()


def test_continuous_batching_trace():
    """Staggered arrivals: queries join lanes while others are in flight."""
    from ipregel_b200 import serve as S
    gs = _graphs()
    dg = _device(gs)
    srv = S.Server(ppr_rounds=20)
    try:
        for d in dg:
            srv.add_graph(d)
        tr = S.poisson_trace(120, 4000.0, [g.V for g in gs], seed=5)
        qids, lat, mk = srv.run_trace(tr, keep_results=True)
        assert mk > 0 and np.all(lat > 0)
        for i in range(len(tr)):
            gid, kind, src = int(tr.gid[i]), int(tr.kind[i]), int(tr.source[i])
            _check(gs[gid], kind, src, srv.result(int(qids[i]), kind, gs[gid].V))
            srv.release(int(qids[i]))
        st = srv.stats()
        assert st["supersteps"] > 0 and st["kernel_launches"] > 0
    finally:
        srv.free()
        for d in dg:
            d.free()


def test_more_queries_than_lanes():
    """100 SSSP queries on one graph: lanes (64) are reused as queries finish."""
    from ipregel_b200 import serve as S
    g = O.add_weights(O.gen_rmat(11, 16, seed=7, undirected=True), wmax=255, seed=7)
    (d,) = _device([g])
    srv = S.Server()
    try:
        gid = srv.add_graph(d)
        srcs = list(range(0, 2000, 20))
        ids = [srv.submit(gid, S.SSSP, s) for s in srcs]
        srv.drain()
        for qid, s in zip(ids, srcs):
            np.testing.assert_array_equal(srv.result(qid, S.SSSP, g.V), O.dijkstra(g, s))
    finally:
        srv.free()
        d.free()


def test_more_ppr_queries_than_lanes():
    """70 PPR queries on one graph: every lane of the group in use at once,
    lanes reused as queries finish; each within the FP32 tolerance of the
    FP64 oracle and bitwise the same as alone."""
    from ipregel_b200 import serve as S
    g = O.add_weights(O.gen_rmat(11, 16, seed=8, undirected=True), wmax=255, seed=8)
    (d,) = _device([g])
    srv = S.Server(ppr_rounds=20)
    try:
        gid = srv.add_graph(d)
        srcs = [int(s) for s in np.random.default_rng(4).integers(0, g.V, size=70)]
        ids = [srv.submit(gid, S.PPR, s) for s in srcs]
        srv.drain()
        got = [srv.result(q, S.PPR, g.V) for q in ids]
        for s, r in zip(srcs, got):
            _check(g, S.PPR, s, r)
        for s, r in list(zip(srcs, got))[::23]:
            alone, _ = S.run_alone(srv, gid, S.PPR, s, g.V)
            np.testing.assert_array_equal(alone.view(np.uint32), r.view(np.uint32))
    finally:
        srv.free()
        d.free()


def test_tight_hbm_budget_evicts_idle_groups():
    from ipregel_b200 import serve as S
    gs = _graphs()
    dg = _device(gs)
    # room for the largest group and its results, not for all groups at once
    V = max(g.V for g in gs)
    budget = V * 300 + 8 * V * 4 + (1 << 20)
    srv = S.Server(hbm_budget=budget)
    try:
        for d in dg:
            srv.add_graph(d)
        qs = [(gid, S.SSSP, 1) for gid in range(3)] + [(gid, S.PPR, 2) for gid in range(3)]
        ids = [srv.submit(*q) for q in qs]
        srv.drain()
        for qid, (gid, kind, src) in zip(ids, qs):
            _check(gs[gid], kind, src, srv.result(qid, kind, gs[gid].V))
        st = srv.stats()
        assert st["peak_bytes"] <= budget
        assert st["groups_freed"] > 0
    finally:
        srv.free()
        for d in dg:
            d.free()


def test_cc_union_find_and_label_propagation():
    """CC on a graph declared symmetric runs by union-find (the labels of
    min-label propagation); on a directed graph by label-propagation lanes."""
    from ipregel_b200 import serve as S
    gs = _graphs()
    dg = _device(gs)
    directed = O.gen_rmat(10, 8, seed=5, undirected=False)
    dd = _device([directed])[0]
    srv = S.Server()
    try:
        for d in dg:
            d.set_symmetric(True)
            srv.add_graph(d)
        gd = srv.add_graph(dd)
        qs = [(gid, S.CC, 0) for gid in range(3) for _ in range(3)] + [(gid, S.SSSP, 5) for gid in range(3)]
        ids = [srv.submit(*q) for q in qs]
        qd = srv.submit(gd, S.CC, 0)
        srv.drain()
        for qid, (gid, kind, src) in zip(ids, qs):
            _check(gs[gid], kind, src, srv.result(qid, kind, gs[gid].V))
        np.testing.assert_array_equal(srv.result(qd, S.CC, directed.V), O.run(directed, "cc", "spread")[0])
    finally:
        srv.free()
        for d in dg + [dd]:
            d.free()


def test_cc_union_find_with_hubs():
    """Union-find on a graph with hub rows split into chunks and a giant
    component whose remaining edges are skipped: the labels of label
    propagation, on two CC queries admitted together."""
    import ipregel_b200 as ip
    from ipregel_b200 import serve as S
    g = O.gen_rmat(16, 16, seed=4, undirected=True)
    d = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    d.set_symmetric(True)
    want = O.run(g, "cc", "spread")[0]
    srv = S.Server()
    try:
        gid = srv.add_graph(d)
        for _ in range(2):
            qs = [srv.submit(gid, S.CC, 0) for _ in range(2)]
            srv.drain()
            for q in qs:
                np.testing.assert_array_equal(srv.result(q, S.CC, g.V), want)
                srv.release(q)
    finally:
        srv.free()
        d.free()


def test_sssp_pull_supersteps_match_push_and_dijkstra():
    """On a graph declared symmetric, dense min-plus supersteps pull (no
    atomics); every distance equals Dijkstra's and the push-only run's."""
    import ipregel_b200 as ip
    from ipregel_b200 import serve as S
    g = O.add_weights(O.gen_rmat(14, 16, seed=11, undirected=True), wmax=255, seed=11)
    srcs = [int(s) for s in np.random.default_rng(3).choice(np.flatnonzero(np.diff(g.idx) > 0), 40, replace=False)]
    results = {}
    for symmetric in (True, False):
        d = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt)
        d.set_symmetric(symmetric)
        srv = S.Server()
        try:
            gid = srv.add_graph(d)
            ids = [srv.submit(gid, S.SSSP, s) for s in srcs]
            srv.drain()
            results[symmetric] = [srv.result(q, S.SSSP, g.V) for q in ids]
            pulls = srv.stats()["pull_supersteps"]
            assert (pulls > 0) if symmetric else (pulls == 0)
        finally:
            srv.free()
            d.free()
    for s, a, b in zip(srcs, results[True], results[False]):
        np.testing.assert_array_equal(a, O.dijkstra(g, s))
        np.testing.assert_array_equal(a, b)


def test_reserved_groups_serve_and_respect_budget():
    """Groups reserved before the queries arrive are the ones the queries run
    in; a reservation that does not fit the budget raises."""
    import ipregel_b200 as ip
    from ipregel_b200 import serve as S
    gs = _graphs()
    dg = _device(gs)
    srv = S.Server()
    try:
        gids = [srv.add_graph(d) for d in dg]
        for gid in gids:
            srv.reserve(gid, S.SSSP)
            srv.reserve(gid, S.PPR)
            srv.reserve(gid, S.SSSP)  # already there: no second group
        st = srv.stats()
        assert st["groups_created"] == 2 * len(gids) and st["bytes_in_use"] > 0
        qs = [(gid, kind, 3) for gid in gids for kind in (S.SSSP, S.PPR)]
        ids = [srv.submit(*q) for q in qs]
        srv.drain()
        for qid, (gid, kind, src) in zip(ids, qs):
            _check(gs[gid], kind, src, srv.result(qid, kind, gs[gid].V))
        assert srv.stats()["groups_created"] == 2 * len(gids)
    finally:
        srv.free()
    small = S.Server(hbm_budget=1 << 20)
    try:
        gid = small.add_graph(dg[2])
        with pytest.raises(ip.IPregelError, match="budget"):
            small.reserve(gid, S.PPR)
    finally:
        small.free()
        for d in dg:
            d.free()


def test_bad_requests_raise():
    import ipregel_b200 as ip
    from ipregel_b200 import serve as S
    g = O.gen_rmat(8, 8, seed=1, undirected=True)
    unweighted = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    srv = S.Server()
    try:
        gid = srv.add_graph(unweighted)
        with pytest.raises(ip.IPregelError, match="weighted"):
            srv.submit(gid, S.SSSP, 0)
        with pytest.raises(ip.IPregelError, match="no such graph"):
            srv.submit(gid + 1, S.CC, 0)
        with pytest.raises(ip.IPregelError, match="out of range"):
            srv.submit(gid, S.PPR, g.V)
        with pytest.raises(ip.IPregelError, match="kind"):
            srv.submit(gid, 7, 0)
        q = srv.submit(gid, S.CC, 0)  # CC needs no weights
        srv.drain()
        np.testing.assert_array_equal(srv.result(q, S.CC, g.V), O.run(g, "cc", "spread")[0])
    finally:
        srv.free()
        unweighted.free()
