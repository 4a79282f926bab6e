"""Parity at the workloads' own sizes.

C1: PageRank (pagerank.c, single_broadcast version, FP64) on the directed
R-MAT graph of scale 16 (edge factor 16, a/b/c = 0.57/0.19/0.19, seed 1),
loaded as pagerank.c loads it (directed = false: the stored rows are the
gather lists, iPregel_postamble.h:368-372), 10 rounds (pagerank.c:34) and
30 rounds (ROUND patched), through the application library and through the
drop-in binaries built from the reference's own pagerank.c; against the
reference's own binaries (oracle/_ref) within 1e-12 max abs per vertex, with
identical per-superstep active counts.

C2: the undirected R-MAT graph of scale 24 (same parameters, weights
U[1,255]): CC and hop-count SSSP from 0 in the spread version bit-exact
against the reference's cc_spread_32 / sssp_spread_32 on the same graph
(combiner_spread_postamble.h:235-342, cc.c:31-55, sssp.c:38-71), their
per-superstep counts identical; weighted SSSP bit-exact against the oracle's
exact Dijkstra, with the pull switch off and on.  Hub rows of 10^5+ edges
take the multi-chunk block classes here, which small graphs never reach."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "ipregel_b200", "bin")
THREADS = str(os.cpu_count() or 4)


def _ref_or_oracle(app, version, g, path, rounds=10):
    """(values, counts) from the reference binary when built, else the oracle."""
    if O.have_ref():
        text, out = O.run_ref(app, version, path, threads=int(THREADS), rounds=rounds, timeout=1800)
        vals = O.parse_dump(app, text, g.V) if app == "pagerank" else O.parse_dump_fast(text, g.V)
        return vals, O.parse_counts(out)
    vals, counts, _ = O.run(g, app, version, rounds=rounds)
    return vals, [int(c) for c in counts]


@pytest.fixture(scope="module")
def c1():
    g = O.gen_rmat(16, 16, seed=1, undirected=False)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "rmat16")
        O.write_graph(g, path)
        yield g, path


@pytest.mark.parametrize("rounds", [10, 30])
def test_c1_pagerank_app_library(c1, rounds):
    import ipregel_b200 as ip
    g, path = c1
    want, want_counts = _ref_or_oracle("pagerank", "single_broadcast", g, path, rounds)
    dg = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)  # directed = false, as pagerank.c loads it
    eng = ip.Engine("pagerank", "single_broadcast")
    try:
        eng.set_quiet(True)
        eng.set_param("rounds", rounds)
        for loop in (False, True):
            eng.set_graph_loop(loop)
            eng.attach(dg)
            res = eng.run()
            assert float(np.max(np.abs(res.values - want))) <= 1e-12
            assert res.counts == want_counts
            assert len(res.counts) == rounds + 1
    finally:
        # parameters are globals of the library: back to pagerank.c's ROUND
        eng.set_param("rounds", 10)
        eng.set_graph_loop(False)
        eng.release()
        dg.free()


@pytest.mark.parametrize("rounds", [10, 30])
def test_c1_pagerank_dropin_binary(c1, rounds):
    g, path = c1
    exe = os.path.join(BIN, "pagerank_r30_single_broadcast_32" if rounds == 30 else "pagerank_single_broadcast_32")
    if not os.path.exists(exe):
        pytest.skip("drop-in binaries not built (make -C ipregel_b200 dropin)")
    want, want_counts = _ref_or_oracle("pagerank", "single_broadcast", g, path, rounds)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.txt")
        p = subprocess.run([exe, path, out, THREADS, "static", "0"], capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        got = O.parse_dump("pagerank", open(out).read(), g.V)
    assert float(np.max(np.abs(got - want))) <= 1e-12
    assert O.parse_counts(p.stdout) == want_counts


@pytest.fixture(scope="module")
def c2():
    import ipregel_b200 as ip
    g = ip.Graph.generate_rmat(24, 16, seed=1, undirected=True, wmax=255)
    idx, adj, wgt = g.to_host()
    host = O.CSR(g.V, g.E, idx, adj, wgt)
    ref = {}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "rmat24")
        g.write(path)
        for app in ("cc", "sssp"):
            ref[app] = _ref_or_oracle(app, "spread", host, path)
    dist = O.dijkstra(host, 0)
    yield g, host, ref, dist
    g.free()


@pytest.mark.parametrize("app", ["cc", "sssp"])
@pytest.mark.parametrize("pull_div", [0, 20])
def test_c2_spread_bit_exact_at_scale_24(c2, app, pull_div):
    import ipregel_b200 as ip
    g, host, ref, _ = c2
    assert g.E > 500_000_000 and host.row_ptr()[1] - host.row_ptr()[0] > 100_000  # hub rows of many chunks
    eng = ip.Engine(app, "spread")
    try:
        eng.set_quiet(True)
        eng.set_tuning(pull_div=pull_div)
        if app == "sssp":
            eng.set_param("source", 0)
        for loop in (True, False):
            eng.set_graph_loop(loop)
            eng.attach(g)
            res = eng.run()
            want, want_counts = ref[app]
            np.testing.assert_array_equal(res.values.astype(np.uint32), want.astype(np.uint32))
            assert res.counts == want_counts
    finally:
        eng.release()


@pytest.mark.parametrize("pull_div", [0, 4, 20])
def test_c2_weighted_sssp_bit_exact_at_scale_24(c2, pull_div):
    import ipregel_b200 as ip
    g, _, _, dist = c2
    eng = ip.Engine("sssp_weighted", "spread")
    try:
        eng.set_quiet(True)
        eng.set_tuning(pull_div=pull_div)
        eng.set_param("source", 0)
        eng.set_graph_loop(True)
        eng.attach(g)
        res = eng.run()
        np.testing.assert_array_equal(res.values, dist)
        # host-driven loop with per-kernel accounting: the pull kernels walked
        # edges exactly when the switch is on
        eng.set_graph_loop(False)
        eng.set_profile(True)
        eng.profile_reset()
        eng.attach(g)
        res = eng.run()
        np.testing.assert_array_equal(res.values, dist)
        pulled = sum(v["edges"] for k, v in eng.profile().items() if k.startswith("pull_deliver"))
        assert (pulled > 0) == (pull_div > 0)
    finally:
        eng.set_profile(False)
        eng.release()
