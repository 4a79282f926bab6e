"""The oracle (oracle/ipregel_oracle.c) against the reference's own OpenMP
binaries (oracle/_ref, built from the reference sources by oracle/Makefile):
identical dumps and identical per-superstep ActiveVertexCount lines."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import small_graphs

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="reference binaries not built (make -C oracle ref)")

APP_VERSIONS = [(a, v) for a in ("cc", "sssp") for v in O.VERSIONS] + \
               [("pagerank", "single_broadcast")]


def _check(g, app, version, threads=2, id_bits=32):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p, id_bytes=id_bits // 8)
        ref_dump, ref_out = O.run_ref(app, version, p, threads=threads, id_bits=id_bits)
    vals, counts, _ = O.run(g, app, version, id_bytes=id_bits // 8)
    assert O.dump_text(app, vals) == ref_dump
    assert list(counts) == O.parse_counts(ref_out)


@pytest.mark.parametrize("app,version", APP_VERSIONS)
@pytest.mark.parametrize("undirected", [True, False])
def test_rmat(app, version, undirected):
    g = O.gen_rmat(11, 16, seed=7, undirected=undirected)
    _check(g, app, version)


@pytest.mark.parametrize("app,version", APP_VERSIONS)
def test_small(app, version):
    for name, g in small_graphs().items():
        if g.V < 2:
            continue  # the reference needs at least as many vertices as threads
        _check(g, app, version, threads=1)


@pytest.mark.parametrize("app,version", [("cc", "combiner"), ("sssp", "spread"), ("cc", "single_broadcast_spread")])
def test_64bit_ids(app, version):
    g = O.gen_rmat(9, 8, seed=3, undirected=True)
    _check(g, app, version, id_bits=64)


def test_pagerank_push_pinned_with_truncation():
    """The push PageRank of the reference truncates the 2nd and later message
    of a mailbox to IP_VERTEX_ID_TYPE (src/combiner_postamble.h:41).  With that
    quirk switched on, the oracle's push engine matches pagerank_32 exactly
    (one thread, so the first message of each mailbox is the first sender's)."""
    g = O.gen_rmat(10, 16, seed=2, undirected=False)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        ref_dump, ref_out = O.run_ref("pagerank", "combiner", p, threads=1)
    vals, counts, _ = O.run(g, "pagerank", "combiner", truncate_push=True)
    assert O.dump_text("pagerank", vals) == ref_dump
    assert list(counts) == O.parse_counts(ref_out)


def test_pagerank_30_rounds():
    g = O.gen_rmat(9, 16, seed=1, undirected=False)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        ref_dump, ref_out = O.run_ref("pagerank", "single_broadcast", p, threads=2, rounds=30)
    vals, counts, _ = O.run(g, "pagerank", "single_broadcast", rounds=30)
    assert O.dump_text("pagerank", vals) == ref_dump
    assert len(counts) == 31


def test_thread_count_does_not_change_reference():
    """Why a sequential restatement suffices: the reference's dumps do not
    depend on the OpenMP team size or schedule for these applications."""
    g = O.gen_rmat(10, 16, seed=5, undirected=True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        O.write_graph(g, p)
        a = O.run_ref("pagerank", "single_broadcast", p, threads=1)[0]
        b = O.run_ref("pagerank", "single_broadcast", p, threads=4, schedule="dynamic", chunk=7)[0]
        c = O.run_ref("cc", "spread", p, threads=1)[0]
        d = O.run_ref("cc", "spread", p, threads=8, schedule="dynamic")[0]
    assert a == b and c == d
