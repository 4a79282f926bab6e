"""Batched many-graph launch.

Many small, independent graphs run as ONE graph: their disjoint union
(ipg_graph_concat: concatenated CSR plus vertex and edge offset tables).  A
vertex-centric program never crosses from one part to another, so one run
over the union gives every part exactly the result it gets alone (CC labels
shifted by the part's vertex offset, which ``split`` removes).  Single-source
SSSP runs from every part's own source at once through the weighted SSSP
application's "batch_offsets" parameter.

Both programs' superstep loops are captured as CUDA graphs with a
device-evaluated while condition and placed in one fused CUDA graph
(``ipregel_b200.Fused``): a whole batch is one launch.  ``autotune`` picks the
CTA size, the degree-class thresholds (threads per vertex) and the push/pull
switch of each program by timing candidate settings on the batch itself.

The plain alternative, one launch loop per graph (``run_plain``), is kept
beside it for comparison and as the equality check.
"""
from __future__ import annotations

import itertools
import time
from dataclasses import dataclass

import numpy as np

from . import DeviceArray, Engine, Fused, Graph

#: Candidate settings of the autotuner: CTA size, (t0, t1) degree-class
#: thresholds (thread per vertex up to t0 edges, warp up to t1, CTAs beyond)
#: and the pull switch (pull when the broadcasters' edges exceed E / pull_div;
#: 0 never pulls).
BLOCKS = (128, 256)
THRESHOLDS = ((8, 1024), (16, 4096), (32, 4096))
PULL_DIVS = (0, 4, 20)


def part_seed(seed: int, i: int) -> int:
    """Generator seed of part i of a batch with base seed `seed`."""
    return int(seed) * 1_000_003 + int(i) + 1


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int = 1) -> np.ndarray:
    """`count` vertex counts log-uniform in [lo, hi] (numpy PCG64, seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.uniform(np.log(lo), np.log(hi), size=count)
    return np.clip(np.floor(np.exp(x)).astype(np.uint64), lo, hi)


def generate_er_parts(sizes, degree=8, seed=1, wmax=64) -> list:
    """Directed Erdos-Renyi parts G(n, degree * n) with weights in
    [1, wmax]; part i uses seed part_seed(seed, i)."""
    return [Graph.generate_er(int(n), int(degree * n), seed=part_seed(seed, i), wmax=wmax)
            for i, n in enumerate(sizes)]


def split_by_offsets(values: np.ndarray, voff: np.ndarray, relabel: bool = False) -> list:
    """Per-part slices of a union's vertex values; relabel subtracts each
    part's vertex offset (for values that are vertex ids, e.g. CC labels)."""
    out = []
    for i in range(len(voff) - 1):
        a, b = int(voff[i]), int(voff[i + 1])
        v = values[a:b]
        out.append((v - v.dtype.type(a)) if relabel else v.copy())
    return out


class Batch:
    """A disjoint union of graphs with its offset tables (host and device)."""

    def __init__(self, parts, directed=True):
        self.parts = list(parts)
        self.union, self.voff, self.eoff = Graph.concat(self.parts, directed=directed)
        self.d_voff = DeviceArray(len(self.voff), np.uint64)
        self.d_voff.from_host(self.voff)

    @property
    def count(self) -> int:
        return len(self.voff) - 1

    def free(self, parts=True):
        self.d_voff.free()
        self.union.free()
        if parts:
            for p in self.parts:
                p.free()
            self.parts = []


@dataclass
class BatchResult:
    cc: list          # per part: CC labels in the part's own ids
    sssp: list        # per part: distances from the part's source
    seconds: float    # device time of the launch
    supersteps: tuple  # (cc, sssp)


class BatchRunner:
    """CC and weighted SSSP over a Batch in one fused CUDA-graph launch."""

    def __init__(self, batch: Batch, source: int = 0, cc_version="spread", sssp_version="spread"):
        self.batch = batch
        self.cc = Engine("cc", cc_version)
        self.sp = Engine("sssp_weighted", sssp_version)
        for e in (self.cc, self.sp):
            e.set_quiet(True)
        self.source = int(source)
        self.tuning = {"cc": dict(block=256, t0=16, t1=4096, pull_div=0),
                       "sssp": dict(block=256, t0=16, t1=4096, pull_div=0)}
        self.fused = None

    def _attach(self, eng, key):
        eng.set_tuning(**self.tuning[key])
        if eng is self.sp:
            eng.set_param("source", self.source)
            eng.set_param_ptr("batch_offsets", self.batch.d_voff.ptr, len(self.batch.voff))
        eng.attach(self.batch.union)

    def prepare(self):
        """Attaches both programs with the current tuning and captures their
        loops into one fused CUDA graph."""
        if self.fused is not None:
            self.fused.free()
        self._attach(self.cc, "cc")
        self._attach(self.sp, "sssp")
        self.fused = Fused()
        self.fused.add(self.cc)
        self.fused.add(self.sp)

    def run(self) -> float:
        if self.fused is None:
            self.prepare()
        return self.fused.run()

    def results(self, seconds=0.0) -> BatchResult:
        cc = split_by_offsets(self.cc.values(), self.batch.voff, relabel=True)
        sp = split_by_offsets(self.sp.values(), self.batch.voff)
        return BatchResult(cc, sp, seconds, (len(self.cc.counts()), len(self.sp.counts())))

    def autotune(self, blocks=BLOCKS, thresholds=THRESHOLDS, pull_divs=PULL_DIVS, reps=2) -> dict:
        """Times every candidate setting of each program on the batch (its own
        captured loop, best of `reps` after one warm-up) and keeps the fastest.
        Returns {program: (setting, seconds)} and leaves the runner prepared."""
        best = {}
        for key, eng in (("cc", self.cc), ("sssp", self.sp)):
            eng.set_graph_loop(True)
            try:
                for block, (t0, t1), pd in itertools.product(blocks, thresholds, pull_divs):
                    self.tuning[key] = dict(block=block, t0=t0, t1=t1, pull_div=pd)
                    self._attach(eng, key)
                    eng.run_only()
                    t = min(self._timed(eng) for _ in range(reps))
                    if key not in best or t < best[key][1]:
                        best[key] = (dict(self.tuning[key]), t)
            finally:
                eng.set_graph_loop(False)
            self.tuning[key] = dict(best[key][0])
        self.prepare()
        return best

    @staticmethod
    def _timed(eng) -> float:
        eng.run_only()
        return eng.stats()[0]

    def release(self):
        if self.fused is not None:
            self.fused.free()
            self.fused = None
        self.sp.set_param_ptr("batch_offsets", None, 0)
        self.cc.release()
        self.sp.release()


def run_plain(parts, source=0, cc_version="spread", sssp_version="spread"):
    """The plain alternative: for every graph, attach and run CC, then SSSP,
    each with the host-driven superstep loop.  Returns (cc, sssp, wall
    seconds, summed device seconds of the loops)."""
    cc = Engine("cc", cc_version)
    sp = Engine("sssp_weighted", sssp_version)
    for e in (cc, sp):
        e.set_quiet(True)
        e.set_graph_loop(False)
        e.set_tuning()
    sp.set_param("source", source)
    sp.set_param_ptr("batch_offsets", None, 0)
    out_cc, out_sp = [], []
    dev = 0.0
    t0 = time.perf_counter()
    for g in parts:
        cc.attach(g)
        cc.run_only()
        out_cc.append(cc.values())
        dev += cc.stats()[0]
        sp.attach(g)
        sp.run_only()
        out_sp.append(sp.values())
        dev += sp.stats()[0]
    wall = time.perf_counter() - t0
    cc.release()
    sp.release()
    return out_cc, out_sp, wall, dev
