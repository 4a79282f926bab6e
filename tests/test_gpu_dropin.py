"""The reference's own applications (benchmarks/cc.c, pagerank.c, sssp.c),
compiled unchanged apart from the qualifier macros against include/iPregel.h
(ipregel_b200/bin/, built by `make -C ipregel_b200 dropin`), run from files
exactly as the reference's binaries are: same argv, same dump format, same
per-superstep log lines."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "ipregel_b200", "bin")

DROPINS = [("cc", v) for v in O.VERSIONS] + [("sssp", v) for v in O.VERSIONS] + \
          [("pagerank", "combiner"), ("pagerank", "single_broadcast")]


def _name(app, version, bits=32, rounds=10):
    base = app + ("_r30" if rounds == 30 else "")
    return os.path.join(BIN, f"{base}{O.VERSION_SUFFIX[version]}_{bits}")


def _run_dropin(exe, graph_path, app):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.txt")
        argv = [exe, graph_path, out, "8", "static", "0"]
        if app == "sssp":
            argv.append("0")
        p = subprocess.run(argv, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        return open(out).read(), p.stdout


@pytest.mark.parametrize("app,version", DROPINS)
@pytest.mark.parametrize("undirected", [True, False])
def test_dropin_binary_matches_reference(app, version, undirected):
    exe = _name(app, version)
    if not os.path.exists(exe):
        pytest.skip("drop-in binaries not built (make -C ipregel_b200 dropin)")
    g = O.gen_rmat(12, 16, seed=3, undirected=undirected)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        dump, out = _run_dropin(exe, p, app)
        ref_dump = ref_counts = None
        if O.have_ref():
            ref_dump, ref_out = O.run_ref(app, version, p, threads=4)
            ref_counts = O.parse_counts(ref_out)
    # pagerank_32 (push) of the reference truncates messages (combiner_postamble.h:41);
    # the GPU push combines in IP_MESSAGE_TYPE, so it is checked against the
    # oracle without the quirk.
    vals, counts, _ = O.run(g, app, version)
    assert O.parse_counts(out) == [int(c) for c in counts]
    if ref_counts is not None:
        assert O.parse_counts(out) == ref_counts
    if app == "pagerank":
        got = O.parse_dump(app, dump, g.V)
        assert np.max(np.abs(got - vals)) <= 1e-12
        if ref_dump is not None and version == "single_broadcast":
            assert np.max(np.abs(got - O.parse_dump(app, ref_dump, g.V))) <= 1e-12
    else:
        assert dump == O.dump_text(app, vals)
        if ref_dump is not None:
            assert dump == ref_dump


def test_dropin_64bit_and_30_rounds():
    for app, version, bits, rounds in (("cc", "combiner", 64, 10), ("sssp", "combiner", 64, 10),
                                       ("pagerank", "single_broadcast", 64, 10),
                                       ("pagerank", "single_broadcast", 32, 30)):
        exe = _name(app, version, bits, rounds)
        if not os.path.exists(exe):
            pytest.skip("drop-in binaries not built")
        g = O.gen_rmat(10, 16, seed=4, undirected=False)
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "g")
            O.write_graph(g, p, id_bytes=bits // 8)
            dump, out = _run_dropin(exe, p, app)
        vals, counts, _ = O.run(g, app, version, id_bytes=bits // 8, rounds=rounds)
        assert O.parse_counts(out) == [int(c) for c in counts]
        if app == "pagerank":
            assert np.max(np.abs(O.parse_dump(app, dump, g.V) - vals)) <= 1e-12
        else:
            assert dump == O.dump_text(app, vals)


def test_dropin_error_paths():
    """Unknown schedule and a missing graph print the reference's message and
    exit with status 255 (exit(-1)), iPregel_postamble.h:188-192 and :139-146."""
    exe = _name("cc", "combiner")
    if not os.path.exists(exe):
        pytest.skip("drop-in binaries not built")
    with tempfile.TemporaryDirectory() as td:
        g = O.gen_rmat(6, 4, seed=1)
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        r = subprocess.run([exe, p, os.path.join(td, "o"), "1", "guided", "0"], capture_output=True, text=True)
        assert r.returncode == 255 and "The schedule guided is unknown." in r.stdout
        r = subprocess.run([exe, os.path.join(td, "nope"), os.path.join(td, "o"), "1", "static", "0"],
                           capture_output=True, text=True)
        assert r.returncode == 255 and "Cannot open the file" in r.stdout
