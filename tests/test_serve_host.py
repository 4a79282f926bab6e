"""Host logic of the request server (no GPU): trace generation and latency
summaries."""
import numpy as np

from ipregel_b200 import serve as S


def test_poisson_trace_shape_and_mix():
    sizes = [1 << 18, 1 << 20, 1 << 25]
    tr = S.poisson_trace(20000, 2000.0, sizes, seed=3)
    assert len(tr) == 20000
    assert np.all(np.diff(tr.arrival) >= 0)
    # mean inter-arrival 1/rate
    assert abs(tr.arrival[-1] / 20000 - 1 / 2000.0) < 0.05 / 2000.0
    frac = [np.mean(tr.kind == k) for k in (S.SSSP, S.PPR, S.CC)]
    assert abs(frac[0] - 0.6) < 0.02 and abs(frac[1] - 0.3) < 0.02 and abs(frac[2] - 0.1) < 0.02
    assert np.all(tr.source < np.asarray(sizes, dtype=np.uint64)[tr.gid])
    assert np.all(tr.source[tr.kind == S.CC] == 0)
    again = S.poisson_trace(20000, 2000.0, sizes, seed=3)
    np.testing.assert_array_equal(tr.arrival, again.arrival)


def test_summarize_percentiles():
    lat = np.linspace(0.001, 0.1, 100)
    kinds = np.array([S.SSSP] * 50 + [S.PPR] * 50)
    s = S.summarize(lat, 2.0, kinds)
    assert s["queries"] == 100 and s["qps"] == 50.0
    assert abs(s["p50_ms"] - np.percentile(lat, 50) * 1e3) < 1e-9
    assert s["p99_ms"] > s["p50_ms"]
    assert "sssp_p99_ms" in s and "ppr_p50_ms" in s and "cc_p50_ms" not in s
