"""The random-gather ceiling (ipg_measure_gather): rates are positive and
finite, a table that fits in L2 serves scattered reads at least as fast as
one that does not, and bad arguments raise instead of launching."""
import math

import pytest

pytestmark = pytest.mark.gpu


def test_gather_rates():
    import ipregel_b200 as ip
    small = ip.measure_gather(16 << 20, 4, 1 << 24, 2)
    large = ip.measure_gather(1 << 30, 4, 1 << 24, 2)
    rows64 = ip.measure_gather(256 << 20, 64, 1 << 22, 2)
    for r in (small, large, rows64):
        assert r["rows_per_s"] > 1e8 and math.isfinite(r["rows_per_s"])
        assert r["gbs"] > 0
    assert small["rows_per_s"] >= 0.9 * large["rows_per_s"]


def test_gather_bad_arguments():
    import ipregel_b200 as ip
    with pytest.raises(ip.IPregelError, match="row_bytes"):
        ip.measure_gather(1 << 20, 8, 1 << 10, 1)
    with pytest.raises(ip.IPregelError, match="table"):
        ip.measure_gather(1 << 20, 4, 0, 1)
