"""Host-side checks of the oracle and of the generators (CPU only)."""
import numpy as np

import oracle as O


def test_rmat_is_deterministic_and_clean():
    a = O.gen_rmat(10, 16, seed=1, undirected=True)
    b = O.gen_rmat(10, 16, seed=1, undirected=True)
    np.testing.assert_array_equal(a.adj, b.adj)
    row = a.row_ptr()
    for v in range(a.V):
        r = a.adj[row[v]:row[v + 1]]
        assert np.all(np.diff(r.astype(np.int64)) > 0)  # sorted, no duplicates
        assert v not in r                                # no self-loops
    # symmetric
    edges = set()
    for v in range(a.V):
        for w in a.adj[row[v]:row[v + 1]]:
            edges.add((v, int(w)))
    assert all((w, v) in edges for (v, w) in edges)


def test_rmat_skew():
    g = O.gen_rmat(12, 16, seed=1, undirected=False)
    deg = np.diff(g.row_ptr().astype(np.int64))
    assert deg[0] == deg.max()  # ids are not permuted: vertex 0 is the top hub
    assert deg.max() > 20 * deg.mean()


def test_weights_symmetric_and_in_range():
    g = O.add_weights(O.gen_rmat(9, 8, seed=2, undirected=True), wmax=255, seed=5)
    row = g.row_ptr()
    w = {}
    for v in range(g.V):
        for e in range(row[v], row[v + 1]):
            w[(v, int(g.adj[e]))] = int(g.wgt[e])
    assert all(1 <= x <= 255 for x in w.values())
    assert all(w[(b, a)] == x for (a, b), x in w.items())


def test_cc_labels_are_component_minima():
    g = O.gen_rmat(11, 4, seed=3, undirected=True)
    vals, _, _ = O.run(g, "cc", "spread")
    # union-find restatement
    parent = list(range(g.V))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    row = g.row_ptr()
    for v in range(g.V):
        for w in g.adj[row[v]:row[v + 1]]:
            a, b = find(v), find(int(w))
            if a != b:
                parent[max(a, b)] = min(a, b)
    comp_min = {}
    for v in range(g.V):
        r = find(v)
        comp_min[r] = min(comp_min.get(r, v), v)
    assert all(vals[v] == comp_min[find(v)] for v in range(g.V))


def test_sssp_hops_match_bfs():
    g = O.gen_rmat(11, 8, seed=4, undirected=True)
    vals, _, _ = O.run(g, "sssp", "combiner")
    row = g.row_ptr()
    dist = np.full(g.V, 0xFFFFFFFF, dtype=np.uint64)
    dist[0] = 0
    frontier = [0]
    while frontier:
        nxt = []
        for v in frontier:
            for w in g.adj[row[v]:row[v + 1]]:
                if dist[w] == 0xFFFFFFFF:
                    dist[w] = dist[v] + 1
                    nxt.append(int(w))
        frontier = nxt
    np.testing.assert_array_equal(vals.astype(np.uint64), dist)


def test_weighted_sssp_versions_equal_dijkstra():
    g = O.add_weights(O.gen_rmat(10, 8, seed=6, undirected=True), wmax=255, seed=6)
    d = O.dijkstra(g, 0)
    for v in ("combiner", "spread"):
        vals, _, _ = O.run(g, "sssp_weighted", v)
        np.testing.assert_array_equal(vals, d)


def test_versions_agree():
    """Cross-version invariant of the reference: all four versions give the
    same CC labels and hop distances."""
    g = O.gen_rmat(10, 16, seed=8, undirected=True)
    for app in ("cc", "sssp"):
        outs = [O.run(g, app, v)[0] for v in O.VERSIONS]
        for o in outs[1:]:
            np.testing.assert_array_equal(o, outs[0])


def test_push_pagerank_equals_pull_on_symmetric_graphs():
    g = O.gen_rmat(10, 16, seed=9, undirected=True)
    a = O.run(g, "pagerank", "combiner")[0]
    b = O.run(g, "pagerank", "single_broadcast")[0]
    assert np.max(np.abs(a - b)) < 1e-15


def test_send_in_single_broadcast_is_an_error():
    g = O.add_weights(O.gen_rmat(6, 4, seed=1, undirected=True), wmax=9)
    import pytest
    with pytest.raises(RuntimeError, match="-3"):
        O.run(g, "sssp_weighted", "single_broadcast")
