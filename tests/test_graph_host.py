"""Host-side argument checks of Graph.refill (no GPU: the checks run before
any call into the runtime)."""
import numpy as np
import pytest

import ipregel_b200 as ip


def _fake_graph(V, E, weight_bytes):
    g = ip.Graph.__new__(ip.Graph)
    g._h = None
    g.view = ip._View()
    g.view.V, g.view.E, g.view.id_bytes, g.view.weight_bytes = V, E, 4, weight_bytes
    return g


def test_refill_checks_sizes_and_weights():
    idx = np.zeros(4, np.uint64)
    adj = np.zeros(6, np.uint32)
    g = _fake_graph(4, 6, 0)
    with pytest.raises(ValueError, match="row starts"):
        g.refill(idx[:3], adj)
    with pytest.raises(ValueError, match="unweighted"):
        g.refill(idx, adj, np.ones(6, np.uint32))
    for wb in (1, 2, 4, 8):
        g = _fake_graph(4, 6, wb)
        with pytest.raises(ValueError, match="weights are required"):
            g.refill(idx, adj)
        with pytest.raises(ValueError, match="expected 6 weights"):
            g.refill(idx, adj, np.ones(5, np.uint64))


def test_weight_dtypes_follow_the_width():
    assert {k: np.dtype(v).itemsize for k, v in ip._WEIGHT_DTYPES.items()} == {1: 1, 2: 2, 4: 4, 8: 8}
