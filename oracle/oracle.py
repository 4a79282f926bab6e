"""ctypes front-end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Wraps ``liboracle.so`` (ipregel_oracle.c, the sequential restatement of the
iPregel superstep engine) and the reference's own binaries in ``oracle/_ref``
(built from the reference sources by ``oracle/Makefile``).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module, and only as the checker; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

VERSIONS = {"combiner": 0, "single_broadcast": 1, "spread": 2, "single_broadcast_spread": 3}
# Binary-name suffix of each version in the reference makefile (makefile:24-27).
VERSION_SUFFIX = {"combiner": "", "spread": "_spread", "single_broadcast": "_single_broadcast",
                  "single_broadcast_spread": "_single_broadcast_spread"}
APPS = {"cc": 0, "pagerank": 1, "sssp": 2, "sssp_weighted": 3, "ppr": 4}


class _Graph(ctypes.Structure):
    _fields_ = [("V", ctypes.c_uint64), ("E", ctypes.c_uint64),
                ("idx", ctypes.c_void_p), ("adj", ctypes.c_void_p), ("wgt", ctypes.c_void_p),
                ("id_bytes", ctypes.c_int), ("directed", ctypes.c_int)]


class _Params(ctypes.Structure):
    _fields_ = [("app", ctypes.c_int), ("version", ctypes.c_int), ("source", ctypes.c_uint64),
                ("rounds", ctypes.c_uint32), ("damping", ctypes.c_double),
                ("truncate_push", ctypes.c_int), ("max_supersteps", ctypes.c_uint64)]


class _Stats(ctypes.Structure):
    _fields_ = [("supersteps", ctypes.c_uint64), ("edges_traversed", ctypes.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
        L = ctypes.CDLL(LIB_PATH)
        L.og_run.restype = ctypes.c_int
        L.og_run.argtypes = [ctypes.POINTER(_Graph), ctypes.POINTER(_Params), ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(_Stats)]
        L.og_gen_rmat.restype = ctypes.c_int64
        L.og_gen_rmat.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_uint64]
        L.og_gen_er.restype = ctypes.c_int64
        L.og_gen_er.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
        L.og_gen_weights.restype = None
        L.og_gen_weights.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p]
        L.og_dijkstra.restype = ctypes.c_int
        L.og_dijkstra.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        L.og_write_graph.restype = ctypes.c_int
        L.og_write_graph.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


@dataclass
class CSR:
    """A graph in the reference loader's layout: idx = V row starts (u64),
    adj = E neighbour ids (u32), wgt = optional E u32 weights."""
    V: int
    E: int
    idx: np.ndarray
    adj: np.ndarray
    wgt: np.ndarray | None = None

    def row_ptr(self) -> np.ndarray:
        return np.append(self.idx, np.uint64(self.E)).astype(np.uint64)


def _finish(V, E, idx, adj):
    return CSR(V, E, idx, adj[:E].copy())


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, undirected=False):
    L = lib()
    V = 1 << scale
    M = (edge_factor << scale) * (2 if undirected else 1)
    idx = np.zeros(V, dtype=np.uint64)
    adj = np.zeros(max(M, 1), dtype=np.uint32)
    E = L.og_gen_rmat(scale, edge_factor, a, b, c, seed, int(undirected), _ptr(idx), _ptr(adj), adj.size)
    if E < 0:
        raise RuntimeError(f"og_gen_rmat failed: {E}")
    return _finish(V, E, idx, adj)


def gen_er(n, m, seed=1, undirected=False):
    L = lib()
    idx = np.zeros(n, dtype=np.uint64)
    adj = np.zeros(max(m * (2 if undirected else 1), 1), dtype=np.uint32)
    E = L.og_gen_er(n, m, seed, int(undirected), _ptr(idx), _ptr(adj), adj.size)
    if E < 0:
        raise RuntimeError(f"og_gen_er failed: {E}")
    return _finish(n, E, idx, adj)


def add_weights(g: CSR, wmax=255, seed=1) -> CSR:
    w = np.zeros(max(g.E, 1), dtype=np.uint32)
    lib().og_gen_weights(g.V, g.E, _ptr(g.idx), _ptr(g.adj), wmax, seed, _ptr(w))
    g.wgt = w[:g.E].copy()
    return g


def from_edges(V, edges, weights=None) -> CSR:
    """CSR from an explicit (src, dst) list, rows in the given order (no
    sorting or dedup, so tests can build any layout the loader accepts)."""
    edges = list(edges)
    rows = [[] for _ in range(V)]
    wrows = [[] for _ in range(V)]
    for k, (s, d) in enumerate(edges):
        rows[s].append(d)
        if weights is not None:
            wrows[s].append(weights[k])
    idx = np.zeros(V, dtype=np.uint64)
    acc = 0
    for v in range(V):
        idx[v] = acc
        acc += len(rows[v])
    adj = np.array([d for r in rows for d in r], dtype=np.uint32)
    wgt = None if weights is None else np.array([w for r in wrows for w in r], dtype=np.uint32)
    return CSR(V, int(acc), idx, adj, wgt)


def run(g: CSR, app: str, version: str, *, source=0, rounds=10, damping=0.85, directed=False,
        id_bytes=4, truncate_push=False, max_supersteps=100000):
    """Runs the restated engine; returns (values, per-superstep active counts)."""
    L = lib()
    adj = g.adj if id_bytes == 4 else g.adj.astype(np.uint64)
    gg = _Graph(g.V, g.E, _ptr(g.idx), _ptr(adj), _ptr(g.wgt), id_bytes, int(directed))
    pp = _Params(APPS[app], VERSIONS[version], source, rounds, damping, int(truncate_push), max_supersteps)
    if app in ("pagerank", "ppr"):
        vals = np.zeros(max(g.V, 1), dtype=np.float64)
    else:
        vals = np.zeros(max(g.V, 1), dtype=np.uint32 if id_bytes == 4 else np.uint64)
    cap = max_supersteps + 1
    counts = np.zeros(cap, dtype=np.uint64)
    st = _Stats()
    rc = L.og_run(ctypes.byref(gg), ctypes.byref(pp), _ptr(vals), _ptr(counts), cap, ctypes.byref(st))
    if rc != 0:
        raise RuntimeError(f"og_run({app}, {version}) failed: {rc}")
    return vals[:g.V], counts[:st.supersteps].copy(), st.edges_traversed


def dijkstra(g: CSR, source=0):
    d = np.zeros(max(g.V, 1), dtype=np.uint32)
    rc = lib().og_dijkstra(g.V, g.E, _ptr(g.idx), _ptr(g.adj), _ptr(g.wgt), source, _ptr(d))
    if rc != 0:
        raise RuntimeError("og_dijkstra failed")
    return d[:g.V]


def write_graph(g: CSR, path: str, id_bytes=4):
    """Writes path.config/.idx/.adj (+ .wgt) in the reference loader format."""
    if id_bytes == 4:
        rc = lib().og_write_graph(path.encode(), g.V, g.E, _ptr(g.idx), _ptr(g.adj), _ptr(g.wgt))
        if rc != 0:
            raise RuntimeError("og_write_graph failed")
    else:
        with open(path + ".config", "w") as f:
            f.write(f"{g.V} {g.E}\n")
        g.idx.astype(np.uint64).tofile(path + ".idx")
        g.adj.astype(np.uint64).tofile(path + ".adj")
        if g.wgt is not None:
            g.wgt.tofile(path + ".wgt")


# ---------------------------------------------------------------------------
# Dumps: the exact text of each app's ip_serialise_vertex.
# ---------------------------------------------------------------------------

def dump_text(app: str, values) -> str:
    """cc.c:65-68 / sssp.c:81-84 print "%u: %u", pagerank.c:73-76 "%lu: %0.20f"."""
    if app in ("pagerank", "ppr"):
        return "".join("%d: %0.20f\n" % (i, float(x)) for i, x in enumerate(values))
    return "".join("%d: %d\n" % (i, int(x) & 0xFFFFFFFF) for i, x in enumerate(values))


def parse_dump(app: str, text: str, V: int):
    if app in ("pagerank", "ppr"):
        out = np.zeros(V, dtype=np.float64)
        for line in text.splitlines():
            k, v = line.split(":")
            out[int(k)] = float(v)
        return out
    out = np.zeros(V, dtype=np.uint64)
    for line in text.splitlines():
        k, v = line.split(":")
        out[int(k)] = int(v)
    return out


_COUNT_RE = re.compile(r"^Superstep(\d+)ActiveVertexCount:(\d+)$", re.M)
_TOTAL_RE = re.compile(r"Total time of supersteps: ([0-9.]+)s\.")


def parse_counts(stdout: str):
    return [int(m.group(2)) for m in _COUNT_RE.finditer(stdout)]


def parse_total_time(stdout: str) -> float:
    m = _TOTAL_RE.search(stdout)
    return float(m.group(1)) if m else float("nan")


def ref_binary(app: str, version: str, id_bits=32, rounds=10) -> str:
    """Path of the reference binary for (app, version) in oracle/_ref."""
    if app == "pagerank" and rounds == 30:
        name = "pagerank_r30" + VERSION_SUFFIX[version] + "_32"
    else:
        name = f"{app}{VERSION_SUFFIX[version]}_{id_bits}"
    return os.path.join(REF_DIR, name)


def have_ref() -> bool:
    return os.path.exists(ref_binary("cc", "combiner"))


def run_ref(app: str, version: str, graph_path: str, *, threads=1, schedule="static", chunk=0,
            id_bits=32, rounds=10, env=None, timeout=600, dump=True):
    """Runs a reference binary on graph files; returns (dump text, stdout).
    dump=False sends the dump to /dev/null and returns "" for it.

    argv follows benchmarks/cc.c:75-81 (sssp.c adds a 6th argument, which it
    ignores: its source vertex is atoi(argv[4]) of the schedule string, i.e. 0,
    sssp.c:94-101)."""
    exe = ref_binary(app, version, id_bits, rounds)
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.txt") if dump else os.devnull
        argv = [exe, graph_path, out, str(threads), schedule, str(chunk)]
        if app == "sssp":
            argv.append("0")
        e = dict(os.environ)
        if env:
            e.update(env)
        p = subprocess.run(argv, capture_output=True, text=True, env=e, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"{exe} failed ({p.returncode}): {p.stdout[-2000:]}")
        if not dump:
            return "", p.stdout
        with open(out) as f:
            return f.read(), p.stdout


def parse_dump_fast(text: str, V: int, dtype=np.uint32):
    """Values of an integer dump ("%u: %u" per line, cc.c:65-68 / sssp.c:81-84)
    in vertex order, vectorised for dumps of millions of lines."""
    nums = np.array(text.replace(":", " ").split(), dtype=np.uint64)
    if nums.size != 2 * V:
        raise ValueError(f"dump has {nums.size // 2} lines, expected {V}")
    ids, vals = nums[0::2], nums[1::2]
    out = np.zeros(V, dtype=dtype)
    out[ids] = vals.astype(dtype)
    if not np.array_equal(np.sort(ids), np.arange(V, dtype=np.uint64)):
        raise ValueError("dump does not list every vertex once")
    return out
