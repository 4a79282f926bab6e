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
def test_reference_run_and_dump_parsing():
    g = O.gen_rmat(12, 16, seed=1, undirected=True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        secs, text, out = bench.reference_run("cc", p, 2, dump=True)
        secs2, text2, _ = bench.reference_run("sssp", p, 2, dump=False)
    assert secs > 0 and secs2 > 0 and text2 is None
    want, counts, _ = O.run(g, "cc", "spread")
    assert (O.parse_dump_fast(text, g.V) == want).all()
    assert O.parse_counts(out) == [int(c) for c in counts]


@pytest.mark.skipif(not O.have_ref(), reason="reference binaries not built")
def test_reference_arm_maps_no_repo_library():
    """The reference arm times the reference's binaries on a graph from the
    oracle's CPU generator: its process maps none of this repository's
    CUDA libraries, and its JSON line names the workload it ran."""
    import json
    import subprocess
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '11', '--steps', '2', "
            "'--warmup', '1']; sys.path.insert(0, %r); import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'mapped': [m for m in ('libipregel_b200', 'app_') if m in maps]}))" % ROOT)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    line, maps = lines[0], lines[1]
    assert maps["mapped"] == []
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert "scale 11" in line["config"]["workload"] and line["cpu_baseline"]["kind"] == "reference"
    assert set(line["per_program"]) == {"cc", "sssp"}


@pytest.mark.skipif(not O.have_ref(), reason="reference binaries not built")
def test_parity_check_against_reference_dumps():
    """bench.parity_check passes results equal to the reference's and the
    oracle's, and fails when one label, one hop distance, one weighted
    distance or one count differs."""
    import numpy as np
    g = O.add_weights(O.gen_rmat(11, 16, seed=2, undirected=True), wmax=255, seed=3)
    dumps = {}
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        for app in ("cc", "sssp"):
            _, text, out = bench.reference_run(app, p, 2, dump=True)
            dumps[app] = (text, out)
    cc, ccn, _ = O.run(g, "cc", "spread")
    hop, hopn, _ = O.run(g, "sssp", "spread")
    w = O.dijkstra(g, 0)
    args = (g.V, g.E, g.idx, g.adj, g.wgt)
    good = bench.parity_check(*args, cc, list(ccn), w, hop, list(hopn), dumps)
    assert good["ok"] and good["cc"]["against"].startswith("reference")
    assert bench.parity_check(*args, cc, list(ccn), w, hop, list(hopn), {})["ok"]  # oracle fallback
    bad_cc = cc.copy()
    bad_cc[5] += 1
    assert not bench.parity_check(*args, bad_cc, list(ccn), w, hop, list(hopn), dumps)["ok"]
    bad_hop = hop.copy()
    bad_hop[-1] ^= 1
    assert not bench.parity_check(*args, cc, list(ccn), w, bad_hop, list(hopn), dumps)["ok"]
    bad_w = w.copy()
    bad_w[np.argmax(w != 0xFFFFFFFF)] += 1
    assert not bench.parity_check(*args, cc, list(ccn), bad_w, hop, list(hopn), dumps)["ok"]
    assert not bench.parity_check(*args, cc, list(ccn)[:-1], w, hop, list(hopn), dumps)["ok"]


def test_traffic_capture_of_other_sources_is_not_used(tmp_path, monkeypatch):
    import json
    p = tmp_path / "traffic.json"
    monkeypatch.setattr(bench, "TRAFFIC_PATH", str(p))
    assert bench.stored_traffic("sssp:push_warp", 1000)["traffic"] is None
    entry = {"dram_bytes_per_algorithmic_byte": 0.5, "source": "capture"}
    p.write_text(json.dumps({"_kernel_sources_sha16": "0" * 16, "sssp:push_warp": entry}))
    r = bench.stored_traffic("sssp:push_warp", 1000)
    assert r["traffic"] is None and "other kernel sources" in r["traffic_source"]
    p.write_text(json.dumps({"_kernel_sources_sha16": bench.kernel_sources_sha16(), "sssp:push_warp": entry}))
    r = bench.stored_traffic("sssp:push_warp", 1000)
    assert r["traffic"] == 500 and r["traffic_source"].startswith("scaled, not measured")


def test_write_traffic_from_launch_list(tmp_path):
    """Launches are assigned to programs by their superstep openers (CC
    first) and to kernels by name; compactions alternate within a superstep."""
    import json
    rows, i = [], 0

    def launch(name, dram):
        nonlocal i
        for metric, v in (("gpu__time_duration.sum", 1000), ("dram__bytes_read.sum", dram),
                          ("dram__bytes_write.sum", 0)):
            rows.append(f'"{i}","1","p","python","0","(1,1,1)","(1,1,1)","{name}","{metric}","byte","{v}"')
        i += 1

    launch("k_generate", 77)  # before the profiled step
    for prog_steps, scale in ((2, 1), (3, 10)):
        for _ in range(prog_steps):
            launch("ipx_k_begin_superstep()", 1)
            launch("ipx_k_compute_spread(const unsigned int *, const unsigned int *)", 2 * scale)
            launch("k_compact(unsigned int *, unsigned long, ...)", 3 * scale)
            launch("void ipx_k_push<1>(const unsigned int *)".replace("void ", ""), 5 * scale)
            launch("k_compact(unsigned int *, unsigned long, ...)", 7 * scale)
    head = ('"ID","Process ID","Process Name","Host Name","Context","Block Size","Grid Size","Kernel Name",'
            '"Metric Name","Metric Unit","Metric Value"')
    csv_path = tmp_path / "l.csv"
    csv_path.write_text("==PROF== x\n" + head + "\n" + "\n".join(rows) + "\n")
    kern = {"cc:compute": {"launches": 2, "bytes": 8}, "sssp:compute": {"launches": 3, "bytes": 60},
            "cc:push_warp": {"launches": 2, "bytes": 20}, "sssp:push_warp": {"launches": 3, "bytes": 300},
            "cc:compact_broadcasters": {"launches": 2, "bytes": 6}, "cc:compact_targets": {"launches": 2, "bytes": 7},
            "sssp:compact_broadcasters": {"launches": 3, "bytes": 90},
            "sssp:compact_targets": {"launches": 3, "bytes": 210}}
    line_path = tmp_path / "line.json"
    line_path.write_text(json.dumps({"kernels": kern, "config": {"scale": 24}}))
    out = bench.write_traffic(str(csv_path), str(line_path), str(tmp_path / "t.json"))
    assert out["_kernel_sources_sha16"] == bench.kernel_sources_sha16()
    assert out["cc:compute"]["dram_bytes_per_algorithmic_byte"] == 0.5  # 2 launches x 2 / 8
    assert out["sssp:push_warp"]["dram_bytes_per_algorithmic_byte"] == 0.5  # 3 x 50 / 300
    assert out["cc:compact_targets"]["dram_bytes_per_algorithmic_byte"] == 2.0  # 2 x 7 / 7
    assert out["sssp:compact_broadcasters"]["launches"] == 3
