"""Request server over resident graphs (ipg_server_*, include/ipregel_b200.h).

Graphs stay in HBM; single-source shortest-path, connected-component and
personalised-PageRank queries run as lanes of fused superstep kernels, with
continuous batching and HBM-budget admission (see ipregel_b200/csrc/serve.cu).
This module wraps the C ABI, generates Poisson query traces, replays them and
summarises latency percentiles and throughput.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import Graph, IPregelError, _check, runtime

SSSP, PPR, CC = 0, 1, 2
KIND_NAMES = {SSSP: "sssp", PPR: "ppr", CC: "cc"}
PENDING, RUNNING, FINISHING, DONE = 0, 1, 2, 3


class _Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "lanes_admitted", "supersteps", "kernel_launches",
                                                 "groups_created", "groups_freed", "bytes_in_use", "peak_bytes",
                                                 "pull_supersteps")]


def _lib():
    L = runtime()
    if not getattr(L, "_serve_typed", False):
        vp, u64, i32, dbl = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
        L.ipg_server_create.argtypes = [u64, ctypes.c_uint32, ctypes.POINTER(vp)]
        L.ipg_server_free.argtypes = [vp]
        L.ipg_server_free.restype = None
        L.ipg_server_add_graph.argtypes = [vp, vp, ctypes.POINTER(i32)]
        L.ipg_server_submit.argtypes = [vp, i32, i32, u64, ctypes.POINTER(u64)]
        L.ipg_server_reserve.argtypes = [vp, i32, i32]
        L.ipg_server_poll.argtypes = [vp, ctypes.POINTER(u64)]
        L.ipg_server_query.argtypes = [vp, u64, ctypes.POINTER(i32), ctypes.POINTER(dbl), ctypes.POINTER(dbl)]
        L.ipg_server_result.argtypes = [vp, u64, vp, u64]
        L.ipg_server_result_device.argtypes = [vp, u64, ctypes.POINTER(vp), ctypes.POINTER(u64)]
        L.ipg_server_release.argtypes = [vp, u64]
        L.ipg_server_get_stats.argtypes = [vp, ctypes.POINTER(_Stats)]
        L.ipg_server_run_trace.argtypes = [vp, u64, vp, vp, vp, vp, i32, vp, vp, ctypes.POINTER(dbl)]
        L.ipg_server_group_stats.argtypes = [vp, i32, i32, ctypes.POINTER(dbl), ctypes.POINTER(u64),
                                             ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L._serve_typed = True
    return L


@dataclass
class Trace:
    """A query arrival trace: arrival times (s, ascending), graph ids, kinds,
    sources."""
    arrival: np.ndarray
    gid: np.ndarray
    kind: np.ndarray
    source: np.ndarray

    def __len__(self):
        return len(self.arrival)


def poisson_trace(n, rate, graph_sizes, mix=(0.6, 0.3, 0.1), seed=1) -> Trace:
    """n queries with Poisson arrivals at `rate` per second; each picks a
    graph uniformly, a kind by `mix` (SSSP, PPR, CC) and a uniform source."""
    rng = np.random.Generator(np.random.PCG64(seed))
    arrival = np.cumsum(rng.exponential(1.0 / rate, size=n))
    gid = rng.integers(0, len(graph_sizes), size=n).astype(np.int32)
    kind = rng.choice(np.array([SSSP, PPR, CC], dtype=np.int32), size=n, p=np.asarray(mix) / np.sum(mix))
    sizes = np.asarray(graph_sizes, dtype=np.uint64)[gid]
    source = (rng.random(n) * sizes).astype(np.uint64)
    source = np.minimum(source, sizes - 1)
    source[kind == CC] = 0
    return Trace(arrival.astype(np.float64), gid, kind.astype(np.int32), source)


def summarize(latency: np.ndarray, makespan: float, kinds=None) -> dict:
    lat = np.asarray(latency, dtype=np.float64)
    out = {"queries": int(lat.size), "makespan_s": makespan, "qps": lat.size / makespan if makespan > 0 else None,
           "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "mean_ms": float(lat.mean() * 1e3)}
    if kinds is not None:
        for k, name in KIND_NAMES.items():
            sel = lat[np.asarray(kinds) == k]
            if sel.size:
                out[f"{name}_p50_ms"] = float(np.percentile(sel, 50) * 1e3)
                out[f"{name}_p99_ms"] = float(np.percentile(sel, 99) * 1e3)
    return out


class Server:
    """ipg_server: resident graphs answering SSSP / PPR / CC queries."""

    def __init__(self, hbm_budget=0, ppr_rounds=20):
        p = ctypes.c_void_p()
        _check(_lib().ipg_server_create(int(hbm_budget), int(ppr_rounds), ctypes.byref(p)), where="ipg_server_create")
        self._p = p
        self.graphs = []
        self.ppr_rounds = ppr_rounds

    def add_graph(self, g: Graph) -> int:
        gid = ctypes.c_int()
        _check(_lib().ipg_server_add_graph(self._p, g.handle, ctypes.byref(gid)), where="ipg_server_add_graph")
        self.graphs.append(g)
        return gid.value

    def reserve(self, gid, kind):
        """Allocates the lane group for queries of `kind` on graph gid now
        (ipg_server_reserve)."""
        _check(_lib().ipg_server_reserve(self._p, int(gid), int(kind)), where="ipg_server_reserve")

    def submit(self, gid, kind, source=0) -> int:
        q = ctypes.c_uint64()
        _check(_lib().ipg_server_submit(self._p, int(gid), int(kind), int(source), ctypes.byref(q)),
               where="ipg_server_submit")
        return q.value

    def poll(self) -> int:
        n = ctypes.c_uint64()
        _check(_lib().ipg_server_poll(self._p, ctypes.byref(n)), where="ipg_server_poll")
        return n.value

    def drain(self):
        while self.poll():
            pass

    def query(self, qid) -> dict:
        st, lat, qd = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        _check(_lib().ipg_server_query(self._p, int(qid), ctypes.byref(st), ctypes.byref(lat), ctypes.byref(qd)),
               where="ipg_server_query")
        return {"state": st.value, "latency": lat.value, "queued": qd.value}

    def result(self, qid, kind, V) -> np.ndarray:
        out = np.empty(V, dtype=np.float32 if kind == PPR else np.uint32)
        _check(_lib().ipg_server_result(self._p, int(qid), out.ctypes.data, out.nbytes), where="ipg_server_result")
        return out

    def release(self, qid):
        _check(_lib().ipg_server_release(self._p, int(qid)), where="ipg_server_release")

    def stats(self) -> dict:
        s = _Stats()
        _check(_lib().ipg_server_get_stats(self._p, ctypes.byref(s)), where="ipg_server_get_stats")
        return {n: getattr(s, n) for n, _ in _Stats._fields_}

    def group_stats(self) -> list:
        """[(gid, "minplus"|"ppr", busy seconds, supersteps, lanes,
        lane-edge relaxations)] of the groups that ran (busy times of
        concurrent groups overlap; relaxations are counted for min-plus)."""
        out = []
        for gid in range(len(self.graphs)):
            for gk, name in ((0, "minplus"), (1, "ppr")):
                b, s, n, w = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
                _check(_lib().ipg_server_group_stats(self._p, gid, gk, ctypes.byref(b), ctypes.byref(s),
                                                     ctypes.byref(n), ctypes.byref(w)), where="ipg_server_group_stats")
                if s.value:
                    out.append((gid, name, b.value, s.value, n.value, w.value))
        return out

    def run_trace(self, trace: Trace, keep_results=False):
        """Replays the trace in real time; returns (qids, latencies s, makespan s)."""
        n = len(trace)
        arr = np.ascontiguousarray(trace.arrival, dtype=np.float64)
        gid = np.ascontiguousarray(trace.gid, dtype=np.int32)
        kind = np.ascontiguousarray(trace.kind, dtype=np.int32)
        src = np.ascontiguousarray(trace.source, dtype=np.uint64)
        qids = np.zeros(n, dtype=np.uint64)
        lat = np.zeros(n, dtype=np.float64)
        mk = ctypes.c_double()
        _check(_lib().ipg_server_run_trace(self._p, n, arr.ctypes.data, gid.ctypes.data, kind.ctypes.data,
                                           src.ctypes.data, int(keep_results), qids.ctypes.data, lat.ctypes.data,
                                           ctypes.byref(mk)), where="ipg_server_run_trace")
        return qids, lat, mk.value

    def free(self):
        if self._p is not None and self._p.value:
            _lib().ipg_server_free(self._p)
        self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def run_alone(srv: Server, gid, kind, source, V):
    """One query with nothing else in flight: its result and latency."""
    q = srv.submit(gid, kind, source)
    srv.drain()
    info = srv.query(q)
    if info["state"] != DONE:
        raise IPregelError("query did not finish")
    r = srv.result(q, kind, V)
    srv.release(q)
    return r, info["latency"]
