"""Host logic of bench.py on CPU: the replica aggregation over ranks (gloo,
world size 2), the clock-record parsing, and the timing of the reference's
binaries on a small sample."""
import os
import sys
import tempfile

import pytest
import torch.multiprocessing as mp

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # each replica timed its own run; the job's time is the slowest rank's
    ms = bench.reduce_max(10.0 + 5.0 * rank, world, "cpu")
    out[rank] = (ms, bench.replica_gteps(world, 1_000_000, 4, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_gloo_two_ranks():
    port = 29500 + (os.getpid() % 1000)
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms, gteps = res[0]
    assert ms == 15.0
    assert gteps == pytest.approx(2 * 1_000_000 * 4 / 0.015 / 1e9)


def test_single_rank_needs_no_process_group():
    assert bench.reduce_max(3.5, 1, "cpu") == 3.5


def test_clock_csv_parsing():
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        f.write("0, 1965, 1965, 700.5, 0x0, Not Active, Not Active, Not Active, Not Active\n")
        f.write("0, 1800, 1965, 990.1, 0x4, Not Active, Not Active, Not Active, Active\n")
        f.write("0, 1700, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active\n")
        f.write("garbage line\n")
        path = f.name
    try:
        c = bench.parse_clock_csv(path)
    finally:
        os.unlink(path)
    assert c["sm_mhz"] == 1800 and c["sm_max_mhz"] == 1965 and c["samples"] == 3
    assert c["reasons"] == ["sw_power_cap"]


def test_nvml_reason_bits():
    import pynvml as n
    assert bench.nvml_reasons(0) == []
    assert bench.nvml_reasons(n.nvmlClocksEventReasonSwPowerCap | n.nvmlClocksEventReasonGpuIdle) == ["sw_power_cap"]
    mask = (n.nvmlClocksEventReasonHwSlowdown | n.nvmlClocksEventReasonSwThermalSlowdown
            | n.nvmlClocksEventReasonHwThermalSlowdown)
    assert sorted(bench.nvml_reasons(mask)) == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_clock_sampler_without_gpu_reports_unavailable():
    s = bench.ClockSampler(0)
    s.start()
    c = s.stop()
    assert "sm_mhz" in c and "reasons" in c


@pytest.mark.skipif(not O.have_ref(), reason="reference binaries not built")
def test_reference_sample_timing():
    g = O.gen_rmat(12, 16, seed=1, undirected=True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        secs, threads = bench.run_reference_sample(p, g.E, 1)
    assert secs > 0 and threads >= 1
