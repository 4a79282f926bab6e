"""Device generators and loaders against the CPU oracle's generators and the
file layout (bit-exact CSR)."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,ef,undirected", [(8, 16, True), (12, 16, False), (14, 16, True), (16, 16, False)])
def test_rmat_matches_cpu(scale, ef, undirected):
    import ipregel_b200 as ip
    want = O.add_weights(O.gen_rmat(scale, ef, seed=1, undirected=undirected), wmax=255, seed=1)
    g = ip.Graph.generate_rmat(scale, ef, seed=1, undirected=undirected, wmax=255)
    idx, adj, wgt = g.to_host()
    assert g.V == want.V and g.E == want.E
    np.testing.assert_array_equal(idx, want.idx)
    np.testing.assert_array_equal(adj, want.adj)
    np.testing.assert_array_equal(wgt, want.wgt)
    g.free()


@pytest.mark.parametrize("n", [1024, 4097, 65536])
def test_er_matches_cpu(n):
    import ipregel_b200 as ip
    want = O.gen_er(n, 8 * n, seed=3)
    g = ip.Graph.generate_er(n, 8 * n, seed=3)
    idx, adj, _ = g.to_host()
    assert g.E == want.E
    np.testing.assert_array_equal(idx, want.idx)
    np.testing.assert_array_equal(adj, want.adj)
    g.free()


def test_file_round_trip_and_in_lists():
    import ipregel_b200 as ip
    want = O.add_weights(O.gen_rmat(11, 16, seed=5, undirected=False), wmax=64, seed=2)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(want, p)
        g = ip.Graph.load(p, directed=True, weighted=True, need_in=True)
        idx, adj, wgt = g.to_host()
        np.testing.assert_array_equal(idx, want.idx)
        np.testing.assert_array_equal(adj, want.adj)
        np.testing.assert_array_equal(wgt, want.wgt)
        # the device writer produces identical files
        p2 = os.path.join(td, "h")
        g.write(p2)
        for ext in (".idx", ".adj", ".wgt", ".config"):
            assert open(p + ext, "rb").read() == open(p2 + ext, "rb").read()
        g.free()


def test_loader_rejects_malformed_files():
    import ipregel_b200 as ip
    g = O.gen_rmat(8, 8, seed=1)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        # truncated adjacency
        with open(p + ".adj", "r+b") as f:
            f.truncate(g.E * 4 - 8)
        with pytest.raises(ip.IPregelError):
            ip.Graph.load(p)
        O.write_graph(g, p)
        # id out of range
        bad = g.adj.copy()
        bad[3] = g.V + 5
        bad.tofile(p + ".adj")
        with pytest.raises(ip.IPregelError):
            ip.Graph.load(p)
        with pytest.raises(ip.IPregelError):
            ip.Graph.load(os.path.join(td, "missing"))


def test_hbm_budget_refuses_cleanly():
    import ipregel_b200 as ip
    g = O.gen_rmat(12, 16, seed=1)
    ip.set_hbm_budget(1 << 16)
    try:
        with pytest.raises(ip.IPregelError, match="budget"):
            ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    finally:
        ip.set_hbm_budget(0)
    gg = ip.Graph.from_csr(g.V, g.E, g.idx, g.adj)
    gg.free()
