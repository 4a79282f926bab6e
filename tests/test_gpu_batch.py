"""Batched many-graph launch: the disjoint union of many ER graphs run as one
fused CUDA-graph launch of CC and weighted SSSP gives every part the result
it gets alone (oracle and plain per-graph loop), under every tuning."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

COUNT, LO, HI, DEG, WMAX = 40, 64, 2048, 8, 64


def _parts(count=COUNT, seed=3):
    from ipregel_b200 import batch as B
    sizes = B.log_uniform_sizes(count, LO, HI, seed=seed)
    return sizes, B.generate_er_parts(sizes, degree=DEG, seed=seed, wmax=WMAX)


def _oracle_part(n, i, seed=3):
    from ipregel_b200 import batch as B
    s = B.part_seed(seed, i)
    return O.add_weights(O.gen_er(int(n), int(DEG * n), seed=s), wmax=WMAX, seed=s)


def test_concat_layout():
    import ipregel_b200 as ip
    sizes, parts = _parts(8)
    u, voff, eoff = ip.Graph.concat(parts, directed=True)
    try:
        idx, adj, wgt = u.to_host()
        for i, p in enumerate(parts):
            pi, pa, pw = p.to_host()
            a, b = int(voff[i]), int(voff[i + 1])
            ea, eb = int(eoff[i]), int(eoff[i + 1])
            np.testing.assert_array_equal(idx[a:b], pi + ea)
            np.testing.assert_array_equal(adj[ea:eb], pa + a)
            np.testing.assert_array_equal(wgt[ea:eb], pw)
        assert u.V == int(voff[-1]) and u.E == int(eoff[-1])
    finally:
        u.free()
        for p in parts:
            p.free()


def test_fused_batch_equals_oracle_per_part():
    from ipregel_b200 import batch as B
    sizes, parts = _parts()
    bt = B.Batch(parts, directed=True)
    r = B.BatchRunner(bt, source=0)
    try:
        sec = r.run()
        res = r.results(sec)
        assert sec > 0
        for i, n in enumerate(sizes):
            g = _oracle_part(n, i)
            want_cc, _, _ = O.run(g, "cc", "spread")
            np.testing.assert_array_equal(res.cc[i], want_cc)
            np.testing.assert_array_equal(res.sssp[i], O.dijkstra(g, 0))
        # a second launch of the same fused graph gives the same results
        r.run()
        again = r.results()
        for i in range(len(sizes)):
            np.testing.assert_array_equal(again.cc[i], res.cc[i])
            np.testing.assert_array_equal(again.sssp[i], res.sssp[i])
    finally:
        r.release()
        bt.free()


def test_batch_equals_plain_loop_under_tunings():
    from ipregel_b200 import batch as B
    sizes, parts = _parts(24, seed=5)
    plain_cc, plain_sp, wall, dev = B.run_plain(parts)
    bt = B.Batch(parts, directed=True)
    r = B.BatchRunner(bt)
    try:
        for tune in (dict(block=128, t0=8, t1=1024, pull_div=0), dict(block=256, t0=32, t1=4096, pull_div=4),
                     dict(block=64, t0=2, t1=64, pull_div=20)):
            r.tuning = {"cc": dict(tune), "sssp": dict(tune)}
            r.prepare()
            res = r.results(r.run())
            for i in range(len(sizes)):
                np.testing.assert_array_equal(res.cc[i], plain_cc[i])
                np.testing.assert_array_equal(res.sssp[i], plain_sp[i])
    finally:
        r.release()
        bt.free(parts=False)
        for p in parts:
            p.free()


def test_autotune_picks_a_candidate_and_keeps_results():
    from ipregel_b200 import batch as B
    sizes, parts = _parts(16, seed=7)
    bt = B.Batch(parts, directed=True)
    r = B.BatchRunner(bt)
    try:
        base = r.results(r.run())
        best = r.autotune(blocks=(128, 256), thresholds=((8, 1024), (16, 4096)), pull_divs=(0, 4), reps=1)
        assert set(best) == {"cc", "sssp"}
        for key, (setting, t) in best.items():
            assert setting["block"] in (128, 256) and t > 0
        res = r.results(r.run())
        for i in range(len(sizes)):
            np.testing.assert_array_equal(res.cc[i], base.cc[i])
            np.testing.assert_array_equal(res.sssp[i], base.sssp[i])
    finally:
        r.release()
        bt.free()


def test_reattached_engine_cannot_run_stale_fused_graph():
    import ipregel_b200 as ip
    from ipregel_b200 import batch as B
    sizes, parts = _parts(4, seed=9)
    bt = B.Batch(parts, directed=True)
    r = B.BatchRunner(bt)
    try:
        r.run()
        r.cc.attach(bt.union)  # the fused graph's cc kernels now hold stale state
        with pytest.raises(ip.IPregelError, match="attached again"):
            r.fused.run()
    finally:
        r.release()
        bt.free()


def test_pull_switch_on_directed_transpose():
    """Push versions on a directed graph with its transpose built may pull
    dense supersteps: same results as pushing."""
    import ipregel_b200 as ip
    g = O.add_weights(O.gen_rmat(12, 16, seed=21, undirected=False), wmax=255, seed=21)
    for app, version in (("cc", "spread"), ("cc", "combiner"), ("sssp_weighted", "spread")):
        graph = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj, wgt=g.wgt, directed=True)
        eng = ip.Engine(app, version)
        eng.set_quiet(True)
        if app.startswith("sssp"):
            eng.set_param("source", 0)
        try:
            eng.set_tuning(pull_div=1_000_000_000)
            eng.attach(graph)
            res = eng.run()
        finally:
            eng.set_tuning()
            eng.release()
            graph.free()
        want, counts, _ = O.run(g, "sssp_weighted" if app.startswith("sssp") else app, version)
        np.testing.assert_array_equal(res.values, want)
        assert res.counts == [int(c) for c in counts]
