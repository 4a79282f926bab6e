#!/usr/bin/env python3
"""Regenerates tests/golden/*.npz: small graphs and the outputs of the
reference's own OpenMP binaries on them (oracle/_ref, built from the reference
sources by `make -C oracle ref`).

Each fixture holds the graph (idx, adj; the loader's layout) and, for every
(application, version) the reference builds, the values parsed from the
reference's dump and its per-superstep ActiveVertexCount lines.  Run from the
repository root:  python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

RUNS = [(a, v) for a in ("cc", "sssp") for v in O.VERSIONS] + [("pagerank", "single_broadcast"),
                                                               ("pagerank", "combiner")]


def graphs():
    return {
        "rmat9_undirected": O.gen_rmat(9, 16, seed=21, undirected=True),
        "rmat10_directed": O.gen_rmat(10, 16, seed=22, undirected=False),
        "er_2000_directed": O.gen_er(2000, 16000, seed=23, undirected=False),
        "two_components": O.from_edges(7, [(0, 1), (1, 0), (1, 2), (2, 1), (3, 4), (4, 3), (4, 5), (5, 4)]),
    }


def main():
    if not O.have_ref():
        sys.exit("reference binaries missing: make -C oracle ref")
    for name, g in graphs().items():
        out = {"V": np.uint64(g.V), "E": np.uint64(g.E), "idx": g.idx, "adj": g.adj}
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "g")
            O.write_graph(g, p)
            for app, version in RUNS:
                # one thread: pagerank_32's truncated mailbox keeps the first
                # sender's message, which is then deterministic
                dump, stdout = O.run_ref(app, version, p, threads=1)
                key = f"{app}__{version}"
                out[key + "__values"] = O.parse_dump(app, dump, g.V)
                out[key + "__counts"] = np.array(O.parse_counts(stdout), dtype=np.uint64)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name, g.V, g.E)


if __name__ == "__main__":
    main()
