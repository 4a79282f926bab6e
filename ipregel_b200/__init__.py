"""iPregel-B200: the iPregel superstep engine on an NVIDIA B200 (sm_100a).

Host-side mirror of the reference's interface for Python callers.  The
reference (a header-only C library) is driven as

    ip_init(path, threads, schedule, chunk, directed, weighted)   # iPregel_preamble.h:298
    ip_run()                                                      # :309
    ip_dump(FILE*)                                                # :317

with one application (ip_compute / ip_combine) compiled in, and the version
chosen at compile time (IP_USE_SPREAD / IP_USE_SINGLE_BROADCAST).  Here each
(application, version, id width) is a prebuilt library ``lib/app_*.so`` that
exports the same ip_* functions plus the ``ipg_app_*`` C ABI; ``Engine`` wraps
one of them, ``Graph`` wraps a device-resident graph of ``libipregel_b200.so``.

There is no CPU path: if the libraries are missing or no GPU is present,
loading raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# IPG_LIB_DIR selects another build of the libraries (e.g. a tuning variant).
LIB_DIR = os.environ.get("IPG_LIB_DIR") or os.path.join(HERE, "lib")
BIN_DIR = os.path.join(HERE, "bin")
RUNTIME_PATH = os.path.join(LIB_DIR, "libipregel_b200.so")

VERSIONS = ("combiner", "spread", "single_broadcast", "single_broadcast_spread")
APPS = ("cc", "sssp", "pagerank", "ppr", "sssp_weighted", "sssp_weighted_send")

# Every symbol of include/ipregel_b200.h.
RUNTIME_SYMBOLS = (
    "ipg_last_error", "ipg_abi_version", "ipg_device_info", "ipg_dev_alloc", "ipg_dev_free",
    "ipg_set_hbm_budget", "ipg_hbm_in_use", "ipg_host_alloc", "ipg_host_free", "ipg_graph_load",
    "ipg_graph_from_host", "ipg_graph_from_device", "ipg_graph_generate_rmat", "ipg_graph_generate_er",
    "ipg_graph_view_get", "ipg_graph_set_symmetric", "ipg_graph_check_symmetric", "ipg_graph_build_in",
    "ipg_graph_to_host", "ipg_graph_write", "ipg_graph_free",
    "ipg_graph_bins", "ipg_degree_classes_noalloc", "ipg_compact", "ipg_bitmap_popc_or", "ipg_sm_count",
    "ipg_graph_set_directed", "ipg_memcpy", "ipg_pr_plan_create", "ipg_pr_plan_free", "ipg_pr_plan_info", "ipg_pr_run_f32",
    "ipg_error_f32_f64", "ipg_graph_concat", "ipg_fused_create", "ipg_fused_graph", "ipg_fused_launch",
    "ipg_fused_free", "ipg_server_create", "ipg_server_free", "ipg_server_add_graph", "ipg_server_submit",
    "ipg_server_poll", "ipg_server_query", "ipg_server_result", "ipg_server_result_device", "ipg_server_release",
    "ipg_server_get_stats", "ipg_server_run_trace", "ipg_server_group_stats",
    "ipg_server_reserve", "ipg_graph_refill_host", "ipg_graph_contents", "ipg_graph_degree_order",
)
# The reference interface (src/iPregel_preamble.h:66-317) and the ipg_app_*
# ABI (include/ipregel_b200/host.cuh), exported by every application library.
APP_SYMBOLS = (
    "ip_get_superstep", "ip_is_first_superstep", "ip_increment_superstep", "ip_set_vertices_count",
    "ip_get_vertices_count", "ip_set_edges_count", "ip_get_edges_count", "ip_get_vertex_by_location",
    "ip_get_vertex_by_id", "ip_init_vertex_range", "ip_load_graph", "ip_safe_malloc", "ip_safe_realloc",
    "ip_safe_free", "ip_safe_fopen", "ip_safe_fread", "ip_safe_fwrite", "ip_init", "ip_init_specific",
    "ip_run", "ip_dump", "ip_serialise_vertex",
    "ipg_app_abi_version", "ipg_app_describe", "ipg_app_last_error", "ipg_app_attach", "ipg_app_load_host",
    "ipg_app_run", "ipg_app_values", "ipg_app_values_device", "ipg_app_supersteps", "ipg_app_counts",
    "ipg_app_stats", "ipg_app_stream", "ipg_app_set_quiet", "ipg_app_set_param", "ipg_app_release",
    "ipg_app_set_profile", "ipg_app_profile_reset", "ipg_app_launches", "ipg_app_profile", "ipg_app_main",
    "ipg_app_set_graph_loop", "ipg_app_graph_loop", "ipg_app_set_tuning", "ipg_app_get_tuning",
    "ipg_app_loop_add", "ipg_app_loop_prepare", "ipg_app_loop_collect", "ipg_app_set_param_ptr",
    "ipg_app_set_order", "ipg_app_order",
)


class IPregelError(RuntimeError):
    pass


class _View(ctypes.Structure):
    _fields_ = [("V", ctypes.c_uint64), ("E", ctypes.c_uint64), ("id_bytes", ctypes.c_int),
                ("weight_bytes", ctypes.c_int), ("directed", ctypes.c_int), ("has_in", ctypes.c_int),
                ("d_row", ctypes.c_void_p), ("d_adj", ctypes.c_void_p), ("d_wgt", ctypes.c_void_p),
                ("d_in_row", ctypes.c_void_p), ("d_in_adj", ctypes.c_void_p), ("d_in_wgt", ctypes.c_void_p),
                ("max_out_degree", ctypes.c_uint64), ("max_in_degree", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64), ("symmetric", ctypes.c_int)]


class _Order(ctypes.Structure):
    _fields_ = [("graph", ctypes.c_void_p), ("d_old_of_new", ctypes.c_void_p), ("d_new_of_old", ctypes.c_void_p)]


def build():
    """Compiles the runtime and the application libraries in-tree (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", HERE, f"-j{os.cpu_count() or 4}"], check=True)


_rt = None


def runtime():
    """Loads libipregel_b200.so (raises if it was not built)."""
    global _rt
    if _rt is None:
        if not os.path.exists(RUNTIME_PATH):
            raise IPregelError(f"{RUNTIME_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(RUNTIME_PATH)
        L.ipg_last_error.restype = ctypes.c_char_p
        L.ipg_hbm_in_use.restype = ctypes.c_uint64
        vp, u64, i32, dbl = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
        L.ipg_graph_from_host.argtypes = [u64, u64, vp, i32, vp, i32, vp, i32, i32, i32, ctypes.POINTER(vp)]
        L.ipg_graph_from_device.argtypes = [u64, u64, vp, vp, i32, vp, i32, i32, i32, ctypes.POINTER(vp)]
        L.ipg_graph_refill_host.argtypes = [vp, vp, i32, vp, vp]
        L.ipg_graph_contents.argtypes = [vp, ctypes.POINTER(u64), ctypes.POINTER(ctypes.c_int)]
        L.ipg_graph_load.argtypes = [ctypes.c_char_p, i32, i32, i32, i32, i32, i32, ctypes.POINTER(vp)]
        L.ipg_graph_generate_rmat.argtypes = [ctypes.c_uint32, ctypes.c_uint32, dbl, dbl, dbl, u64, i32,
                                              ctypes.c_uint32, i32, ctypes.POINTER(vp)]
        L.ipg_graph_generate_er.argtypes = [u64, u64, u64, i32, ctypes.c_uint32, i32, ctypes.POINTER(vp)]
        L.ipg_graph_view_get.argtypes = [vp, ctypes.POINTER(_View)]
        L.ipg_graph_build_in.argtypes = [vp]
        L.ipg_graph_degree_order.argtypes = [vp, i32, ctypes.POINTER(_Order)]
        L.ipg_graph_set_symmetric.argtypes = [vp, i32]
        L.ipg_graph_set_directed.argtypes = [vp, i32]
        L.ipg_graph_check_symmetric.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.ipg_graph_to_host.argtypes = [vp, vp, vp, vp]
        L.ipg_graph_write.argtypes = [vp, ctypes.c_char_p]
        L.ipg_graph_free.argtypes = [vp]
        L.ipg_graph_free.restype = None
        L.ipg_dev_alloc.argtypes = [ctypes.POINTER(vp), u64]
        L.ipg_dev_free.argtypes = [vp, u64]
        L.ipg_host_alloc.argtypes = [ctypes.POINTER(vp), u64]
        L.ipg_host_free.argtypes = [vp]
        L.ipg_set_hbm_budget.argtypes = [u64]
        L.ipg_device_info.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(u64),
                                      ctypes.POINTER(ctypes.c_int)]
        L.ipg_memcpy.argtypes = [vp, vp, u64]
        L.ipg_graph_concat.argtypes = [vp, ctypes.c_uint32, i32, i32, ctypes.POINTER(vp), vp, vp]
        L.ipg_fused_create.argtypes = [ctypes.POINTER(vp)]
        L.ipg_fused_graph.argtypes = [vp]
        L.ipg_fused_graph.restype = vp
        L.ipg_fused_launch.argtypes = [vp, vp, ctypes.POINTER(dbl)]
        L.ipg_fused_free.argtypes = [vp]
        L.ipg_fused_free.restype = None
        L.ipg_pr_plan_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.ipg_pr_plan_free.argtypes = [vp]
        L.ipg_pr_plan_free.restype = None
        L.ipg_pr_plan_info.argtypes = [vp, vp, vp, vp]
        L.ipg_pr_run_f32.argtypes = [vp, ctypes.c_uint32, dbl, i32, vp, vp, vp]
        L.ipg_error_f32_f64.argtypes = [vp, vp, u64, ctypes.POINTER(dbl), ctypes.POINTER(dbl),
                                        ctypes.POINTER(dbl), ctypes.POINTER(u64), vp]
        _rt = L
    return _rt


def _check(rc, lib=None, where=""):
    if rc != 0:
        msg = (lib or runtime()).ipg_last_error()
        msg = msg.decode() if isinstance(msg, bytes) else str(msg)
        raise IPregelError(f"{where} failed ({rc}): {msg}")


def device_info():
    name = ctypes.create_string_buffer(256)
    hbm = ctypes.c_uint64()
    sms = ctypes.c_int()
    _check(runtime().ipg_device_info(name, 256, ctypes.byref(hbm), ctypes.byref(sms)), where="ipg_device_info")
    return {"name": name.value.decode(), "hbm_bytes": hbm.value, "sm_count": sms.value}


def set_hbm_budget(nbytes: int):
    runtime().ipg_set_hbm_budget(int(nbytes))


def hbm_in_use() -> int:
    return int(runtime().ipg_hbm_in_use())


class PinnedArray:
    """A numpy array over page-locked host memory (for host<->device copies
    inside timed regions)."""

    def __init__(self, n, dtype):
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        p = ctypes.c_void_p()
        _check(runtime().ipg_host_alloc(ctypes.byref(p), max(self.n * self.dtype.itemsize, 16)),
               where="ipg_host_alloc")
        self._p = p
        buf = (ctypes.c_char * max(self.n * self.dtype.itemsize, 16)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=self.n)

    @property
    def ptr(self):
        return self._p.value

    def free(self):
        if self._p is not None and self._p.value:
            runtime().ipg_host_free(self._p)
        self._p = None
        self.array = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class DeviceArray:
    """n elements of dtype in HBM, allocated through the runtime's budgeted
    allocator (ipg_dev_alloc)."""

    def __init__(self, n, dtype):
        self.dtype = np.dtype(dtype)
        self.n = int(n)
        self.nbytes = max(self.n * self.dtype.itemsize, 16)
        self._owned = True
        p = ctypes.c_void_p()
        _check(runtime().ipg_dev_alloc(ctypes.byref(p), self.nbytes), where="ipg_dev_alloc")
        self._p = p

    @classmethod
    def wrap(cls, ptr, n, dtype):
        """A view of device memory owned elsewhere (free() leaves it alone)."""
        a = cls.__new__(cls)
        a.dtype, a.n = np.dtype(dtype), int(n)
        a.nbytes = a.n * a.dtype.itemsize
        a._owned = False
        a._p = ctypes.c_void_p(ptr)
        return a

    @property
    def ptr(self):
        return self._p.value

    def to_host(self):
        out = np.empty(self.n, dtype=self.dtype)
        if self.n:
            _check(runtime().ipg_memcpy(out.ctypes.data, self._p, self.n * self.dtype.itemsize), where="ipg_memcpy")
        return out

    def from_host(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        assert a.size == self.n
        if self.n:
            _check(runtime().ipg_memcpy(self._p, a.ctypes.data, self.n * self.dtype.itemsize), where="ipg_memcpy")

    def free(self):
        if self._p is not None and self._p.value and self._owned:
            runtime().ipg_dev_free(self._p, ctypes.c_uint64(self.nbytes))
        self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


_WEIGHT_DTYPES = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


class Graph:
    """A graph resident in HBM (the reference loader's CSR,
    src/iPregel_postamble.h:244-421, plus the in-CSR when needed)."""

    def __init__(self, handle):
        self._h = handle
        self.view = _View()
        _check(runtime().ipg_graph_view_get(handle, ctypes.byref(self.view)), where="ipg_graph_view_get")

    @property
    def handle(self):
        return self._h

    @property
    def V(self):
        return int(self.view.V)

    @property
    def E(self):
        return int(self.view.E)

    def refresh(self):
        _check(runtime().ipg_graph_view_get(self._h, ctypes.byref(self.view)), where="ipg_graph_view_get")

    def degree_order(self, need_in=False) -> dict:
        """The degree-ordered copy the engine runs on (ipg_graph_degree_order),
        read back to the host: old_of_new, new_of_old, the copy's row / adj /
        wgt and, when it has in-lists, in_row / in_adj."""
        rt = runtime()
        o = _Order()
        _check(rt.ipg_graph_degree_order(self._h, int(need_in), ctypes.byref(o)), where="ipg_graph_degree_order")
        V = self.V
        view = _View()
        _check(rt.ipg_graph_view_get(o.graph, ctypes.byref(view)), where="ipg_graph_view_get")
        idt = np.uint32 if view.id_bytes == 4 else np.uint64
        out = {"old_of_new": DeviceArray.wrap(o.d_old_of_new, V, np.uint32).to_host(),
               "new_of_old": DeviceArray.wrap(o.d_new_of_old, V, np.uint32).to_host(),
               "row": DeviceArray.wrap(view.d_row, V + 1, np.uint64).to_host(),
               "adj": DeviceArray.wrap(view.d_adj, view.E, idt).to_host(),
               "wgt": (DeviceArray.wrap(view.d_wgt, view.E, _WEIGHT_DTYPES[int(view.weight_bytes)]).to_host()
                       if view.d_wgt else None),
               "has_in": bool(view.has_in), "in_alias": bool(view.has_in and view.d_in_row == view.d_row)}
        if view.has_in:
            out["in_row"] = DeviceArray.wrap(view.d_in_row, V + 1, np.uint64).to_host()
            out["in_adj"] = DeviceArray.wrap(view.d_in_adj, view.E, idt).to_host()
        return out

    @classmethod
    def from_csr(cls, V, E, idx, adj, wgt=None, directed=False, need_in=False, id_bytes=4):
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        adj = np.ascontiguousarray(adj, dtype=np.uint32 if id_bytes == 4 else np.uint64)
        if wgt is not None:
            wgt = np.ascontiguousarray(wgt, dtype=np.uint32)
        h = ctypes.c_void_p()
        rc = runtime().ipg_graph_from_host(int(V), int(E), idx.ctypes.data if V else None, 8,
                                           adj.ctypes.data if E else None, id_bytes,
                                           wgt.ctypes.data if (wgt is not None and E) else None,
                                           4 if wgt is not None else 0, int(directed), int(need_in),
                                           ctypes.byref(h))
        _check(rc, where="ipg_graph_from_host")
        return cls(h.value)

    def refill(self, idx, adj, wgt=None):
        """New contents of the same size from host buffers, into this graph's
        device buffers (ipg_graph_refill_host): nothing is allocated.  The
        symmetric declaration and other derived data are dropped."""
        V, E = int(self.view.V), int(self.view.E)
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        adj = np.ascontiguousarray(adj, dtype=np.uint32 if int(self.view.id_bytes) == 4 else np.uint64)
        if idx.size != V or adj.size != E:
            raise ValueError(f"refill: expected {V} row starts and {E} ids, got {idx.size} and {adj.size}")
        wb = int(self.view.weight_bytes)
        if wb == 0:
            if wgt is not None:
                raise ValueError("refill: the graph is unweighted, but weights were given")
        else:
            if wgt is None:
                if E:
                    raise ValueError(f"refill: the graph is weighted ({wb}-byte weights): weights are required")
            else:
                wgt = np.ascontiguousarray(wgt, dtype=_WEIGHT_DTYPES[wb])
                if wgt.size != E:
                    raise ValueError(f"refill: expected {E} weights, got {wgt.size}")
        _check(runtime().ipg_graph_refill_host(self._h, idx.ctypes.data if V else None, 8,
                                               adj.ctypes.data if E else None,
                                               wgt.ctypes.data if (wgt is not None and E) else None),
               where="ipg_graph_refill_host")
        self.refresh()

    def contents(self):
        """(generation, valid): the contents generation (+1 at every refill)
        and whether the last refill passed validation (ipg_graph_contents)."""
        gen = ctypes.c_uint64()
        ok = ctypes.c_int()
        _check(runtime().ipg_graph_contents(self._h, ctypes.byref(gen), ctypes.byref(ok)), where="ipg_graph_contents")
        return int(gen.value), bool(ok.value)

    @classmethod
    def generate_rmat(cls, scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, undirected=False, wmax=0,
                      need_in=False):
        h = ctypes.c_void_p()
        _check(runtime().ipg_graph_generate_rmat(scale, edge_factor, a, b, c, seed, int(undirected), wmax,
                                                 int(need_in), ctypes.byref(h)), where="ipg_graph_generate_rmat")
        return cls(h.value)

    @classmethod
    def concat(cls, parts, directed=False, need_in=False):
        """Disjoint union (ipg_graph_concat): (graph, vertex offsets, edge
        offsets), the offsets with len(parts) + 1 entries."""
        n = len(parts)
        arr = (ctypes.c_void_p * n)(*[p.handle for p in parts])
        voff = np.zeros(n + 1, dtype=np.uint64)
        eoff = np.zeros(n + 1, dtype=np.uint64)
        h = ctypes.c_void_p()
        _check(runtime().ipg_graph_concat(arr, n, int(directed), int(need_in), ctypes.byref(h), voff.ctypes.data,
                                          eoff.ctypes.data), where="ipg_graph_concat")
        return cls(h.value), voff, eoff

    @classmethod
    def generate_er(cls, n, m, seed=1, undirected=False, wmax=0, need_in=False):
        h = ctypes.c_void_p()
        _check(runtime().ipg_graph_generate_er(n, m, seed, int(undirected), wmax, int(need_in), ctypes.byref(h)),
               where="ipg_graph_generate_er")
        return cls(h.value)

    @classmethod
    def load(cls, path, id_bytes=4, idx_bytes=8, directed=False, weighted=False, weight_bytes=4, need_in=False):
        h = ctypes.c_void_p()
        _check(runtime().ipg_graph_load(path.encode(), id_bytes, idx_bytes, int(directed), int(weighted),
                                        weight_bytes, int(need_in), ctypes.byref(h)), where="ipg_graph_load")
        return cls(h.value)

    @property
    def symmetric(self) -> bool:
        return bool(self.view.symmetric)

    def set_symmetric(self, symmetric=True):
        """Declares the stored graph symmetric (weights included), which lets
        the push versions pull in dense supersteps.  A wrong declaration gives
        wrong results; check_symmetric() verifies it on the device."""
        _check(runtime().ipg_graph_set_symmetric(self._h, int(symmetric)), where="ipg_graph_set_symmetric")
        self.refresh()

    def set_directed(self, directed=True):
        """ip_init's `directed` for a resident graph: False makes the in-lists
        alias the rows (the reference's benchmarks), True the transpose."""
        _check(runtime().ipg_graph_set_directed(self._h, int(directed)), where="ipg_graph_set_directed")
        self.refresh()

    def check_symmetric(self) -> int:
        """1 symmetric, 0 not, -1 rows not sorted (cannot tell)."""
        r = ctypes.c_int()
        _check(runtime().ipg_graph_check_symmetric(self._h, ctypes.byref(r)), where="ipg_graph_check_symmetric")
        return r.value

    def build_in(self):
        _check(runtime().ipg_graph_build_in(self._h), where="ipg_graph_build_in")
        self.refresh()

    def to_host(self):
        """(idx, adj, wgt) numpy arrays in the file layout."""
        V, E = self.V, self.E
        idx = np.zeros(max(V, 1), dtype=np.uint64)
        adj = np.zeros(max(E, 1), dtype=np.uint32 if self.view.id_bytes == 4 else np.uint64)
        wgt = np.zeros(max(E, 1), dtype=_WEIGHT_DTYPES[int(self.view.weight_bytes)]) if self.view.d_wgt else None
        _check(runtime().ipg_graph_to_host(self._h, idx.ctypes.data, adj.ctypes.data,
                                           wgt.ctypes.data if wgt is not None else None), where="ipg_graph_to_host")
        return idx[:V], adj[:E], (wgt[:E] if wgt is not None else None)

    def write(self, path):
        _check(runtime().ipg_graph_write(self._h, path.encode()), where="ipg_graph_write")

    def free(self):
        if self._h:
            runtime().ipg_graph_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


@dataclass
class RunResult:
    values: np.ndarray
    counts: list = field(default_factory=list)   # per-superstep ActiveVertexCount
    seconds: float = 0.0                         # sum of per-superstep device times
    edges: int = 0                               # edges traversed by the engine
    supersteps: int = 0


def app_library(app: str, version: str, id_bits: int = 32, generic: bool = False, variant: str = "") -> str:
    """Path of an application library; `variant` names a build of other
    kernel switches ("staged": the pull gather's hub chunks a CTA each, ids
    staged in shared memory)."""
    prefix = "appgeneric" if generic else f"app{variant}"
    return os.path.join(LIB_DIR, f"{prefix}_{app}_{version}_{id_bits}.so")


class Engine:
    """One application compiled in one version: the ip_init / ip_run / ip_dump
    life cycle of the reference, on in-memory graphs."""

    _loaded = {}
    # attach generation of every library: a fused launch captured under one
    # attach must not run after another (its kernels hold the old state)
    _generation = {}

    def __init__(self, app: str, version: str = "combiner", id_bits: int = 32, generic: bool = False,
                 variant: str = ""):
        if version not in VERSIONS:
            raise ValueError(f"unknown version {version!r}; expected one of {VERSIONS}")
        path = app_library(app, version, id_bits, generic, variant)
        if not os.path.exists(path):
            raise IPregelError(f"{path} is missing: build it with `make -C {HERE}`")
        runtime()
        if path not in Engine._loaded:
            L = ctypes.CDLL(path)
            vp, u64 = ctypes.c_void_p, ctypes.c_uint64
            L.ipg_app_last_error.restype = ctypes.c_char_p
            L.ipg_app_attach.argtypes = [vp]
            L.ipg_app_load_host.argtypes = [u64, u64, vp, vp, vp, ctypes.c_int]
            L.ipg_app_values.argtypes = [vp, u64]
            L.ipg_app_values_device.argtypes = [ctypes.POINTER(vp)]
            L.ipg_app_supersteps.restype = u64
            L.ipg_app_counts.argtypes = [vp, u64]
            L.ipg_app_stats.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(u64), ctypes.POINTER(u64)]
            L.ipg_app_stream.restype = vp
            L.ipg_app_set_param.argtypes = [ctypes.c_char_p, ctypes.c_double]
            L.ipg_app_describe.argtypes = [ctypes.c_char_p, ctypes.c_int]
            L.ipg_app_release.restype = None
            L.ip_get_vertices_count.restype = ctypes.c_size_t
            L.ipg_app_launches.restype = u64
            L.ipg_app_profile.argtypes = [ctypes.c_char_p, ctypes.c_int]
            L.ipg_app_profile_reset.restype = None
            L.ipg_app_set_tuning.argtypes = [ctypes.c_int, u64, u64, u64]
            L.ipg_app_get_tuning.argtypes = [vp, vp, vp, vp]
            L.ipg_app_loop_add.argtypes = [vp]
            L.ipg_app_loop_collect.argtypes = [ctypes.c_double]
            L.ipg_app_set_param_ptr.argtypes = [ctypes.c_char_p, vp, u64]
            Engine._loaded[path] = L
        self.lib = Engine._loaded[path]
        self.path = path
        self.app, self.version, self.id_bits = app, version, id_bits
        self.info = self.describe()
        self.graph = None

    def describe(self) -> dict:
        buf = ctypes.create_string_buffer(512)
        self.lib.ipg_app_describe(buf, 512)
        return dict(kv.split("=", 1) for kv in buf.value.decode().split())

    def _check(self, rc, where):
        if rc != 0:
            raise IPregelError(f"{where} failed ({rc}): {self.lib.ipg_app_last_error().decode()}")

    @property
    def value_dtype(self):
        kind, nbytes = self.info["value_kind"], int(self.info["value_bytes"])
        return np.dtype({"f": "f", "i": "i", "u": "u"}[kind] + str(nbytes))

    def set_quiet(self, quiet=True):
        self.lib.ipg_app_set_quiet(int(quiet))

    def set_param(self, key, value):
        self._check(self.lib.ipg_app_set_param(key.encode(), float(value)), f"set_param({key})")

    def _bump(self):
        Engine._generation[self.path] = Engine._generation.get(self.path, 0) + 1

    @property
    def generation(self) -> int:
        return Engine._generation.get(self.path, 0)

    def attach(self, graph: Graph):
        self.graph = graph
        self._bump()
        self._check(self.lib.ipg_app_attach(graph.handle), "ipg_app_attach")

    def load_host(self, V, E, idx, adj, wgt=None, directed=False):
        """ip_init from host buffers (idx = V row starts, u64; adj = ids)."""
        self.graph = None
        self._bump()
        self._check(self.lib.ipg_app_load_host(int(V), int(E), _ptr(idx), _ptr(adj), _ptr(wgt), int(directed)),
                    "ipg_app_load_host")

    def run_only(self):
        self._check(self.lib.ipg_app_run(), "ipg_app_run")

    def vertex_count(self) -> int:
        return int(self.lib.ip_get_vertices_count())

    def values(self, out=None):
        """Copies the vertex values to the host (the data ip_dump serialises)."""
        n = self.vertex_count()
        if out is None:
            out = np.zeros(max(n, 1), dtype=self.value_dtype)
        self._check(self.lib.ipg_app_values(_ptr(out), out.nbytes), "ipg_app_values")
        return out[:n] if isinstance(out, np.ndarray) else out

    def counts(self):
        n = int(self.lib.ipg_app_supersteps())
        buf = np.zeros(max(n, 1), dtype=np.uint64)
        self.lib.ipg_app_counts(buf.ctypes.data, n)
        return [int(x) for x in buf[:n]]

    def stats(self):
        s = ctypes.c_double()
        e = ctypes.c_uint64()
        n = ctypes.c_uint64()
        self.lib.ipg_app_stats(ctypes.byref(s), ctypes.byref(e), ctypes.byref(n))
        return s.value, int(e.value), int(n.value)

    def stream(self):
        return self.lib.ipg_app_stream()

    def set_profile(self, on=True):
        self._check(self.lib.ipg_app_set_profile(int(on)), "ipg_app_set_profile")

    def profile_reset(self):
        self.lib.ipg_app_profile_reset()

    def set_graph_loop(self, on=True):
        """Run supersteps as one captured CUDA graph whose while condition is
        evaluated on the device (no host synchronisation per superstep)."""
        self._check(self.lib.ipg_app_set_graph_loop(int(on)), "ipg_app_set_graph_loop")

    def graph_loop(self) -> bool:
        return bool(self.lib.ipg_app_graph_loop())

    def set_order(self, on=True):
        """Run the kernels on the graph's degree-ordered copy (the default)
        or on its own numbering; applied at the next attach.  Results are
        the same either way."""
        self._check(self.lib.ipg_app_set_order(int(on)), "ipg_app_set_order")

    def order(self) -> bool:
        """Whether the attached graph runs renamed."""
        return bool(self.lib.ipg_app_order())

    def set_tuning(self, block=256, t0=16, t1=4096, pull_div=0):
        """CTA size, degree-class thresholds and pull switch of the superstep
        kernels; applied at the next attach."""
        self._check(self.lib.ipg_app_set_tuning(int(block), int(t0), int(t1), int(pull_div)), "ipg_app_set_tuning")

    def tuning(self) -> dict:
        b = ctypes.c_int()
        t0, t1, pd = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.ipg_app_get_tuning(ctypes.byref(b), ctypes.byref(t0), ctypes.byref(t1), ctypes.byref(pd))
        return {"block": b.value, "t0": t0.value, "t1": t1.value, "pull_div": pd.value}

    def set_param_ptr(self, key, ptr, n):
        """A named device array (e.g. "batch_offsets" of weighted SSSP)."""
        self._check(self.lib.ipg_app_set_param_ptr(key.encode(), ptr, int(n)), f"set_param_ptr({key})")

    def loop_add(self, fused: "Fused"):
        """Adds this engine's captured superstep loop to a fused launch."""
        self._check(self.lib.ipg_app_loop_add(fused.cuda_graph), "ipg_app_loop_add")

    def loop_prepare(self):
        self._check(self.lib.ipg_app_loop_prepare(), "ipg_app_loop_prepare")

    def loop_collect(self, seconds: float):
        self._check(self.lib.ipg_app_loop_collect(float(seconds)), "ipg_app_loop_collect")

    def launches(self) -> int:
        """Kernel launches of this application library since the last reset."""
        return int(self.lib.ipg_app_launches())

    def profile(self) -> dict:
        """{kernel: {launches, timed, ms, bytes, edges}} accumulated while
        profiling; edges = edges walked by push, mark and gather kernels."""
        buf = ctypes.create_string_buffer(8192)
        self.lib.ipg_app_profile(buf, 8192)
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, t, ms, b, e = line.split()
            out[name] = {"launches": int(n), "timed": int(t), "ms": float(ms), "bytes": float(b), "edges": float(e)}
        return out

    def run(self) -> RunResult:
        self.run_only()
        vals = self.values()
        sec, edges, n = self.stats()
        return RunResult(vals, self.counts(), sec, edges, n)

    def release(self):
        self._bump()
        self.lib.ipg_app_release()
        self.graph = None

    def main(self, argv):
        """Calls the application's own main (ip_init from files, ip_run,
        ip_dump) in this process."""
        args = [a.encode() for a in argv]
        arr = (ctypes.c_char_p * (len(args) + 1))(*args, None)
        self.lib.ipg_app_main.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        return self.lib.ipg_app_main(len(args), arr)


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, PinnedArray):
        return a.ptr
    return a.ctypes.data


def run_app(app, version, graph: Graph, id_bits=32, params=None, generic=False, quiet=True,
            graph_loop=None, order=None) -> RunResult:
    """Attach + set params + run, returning values and per-superstep counts.
    graph_loop: None keeps the library's mode (IPG_GRAPH_LOOP), True/False
    selects the captured or the host-driven superstep loop; order: None
    keeps the library's mode, True/False runs on the degree-ordered copy or
    on the graph's own numbering (both modes are library-wide and stay set)."""
    eng = Engine(app, version, id_bits, generic)
    eng.set_quiet(quiet)
    if graph_loop is not None:
        eng.set_graph_loop(graph_loop)
    if order is not None:
        eng.set_order(order)
    for k, v in (params or {}).items():
        eng.set_param(k, v)
    eng.attach(graph)
    return eng.run()


class Fused:
    """One CUDA graph holding several engines' captured superstep loops
    (ipg_fused_*): loop_add each engine, then run()."""

    def __init__(self):
        p = ctypes.c_void_p()
        _check(runtime().ipg_fused_create(ctypes.byref(p)), where="ipg_fused_create")
        self._p = p
        self.engines = []

    @property
    def cuda_graph(self):
        return runtime().ipg_fused_graph(self._p)

    def add(self, engine: "Engine"):
        engine.loop_add(self)
        self.engines.append((engine, engine.generation))

    def run(self, stream=None) -> float:
        """prepare, one launch, collect; returns the launch's device seconds."""
        for e, gen in self.engines:
            if e.generation != gen:
                raise IPregelError(f"{e.app}/{e.version} was attached again after it joined this fused launch")
        for e, _ in self.engines:
            e.loop_prepare()
        sec = ctypes.c_double()
        _check(runtime().ipg_fused_launch(self._p, stream, ctypes.byref(sec)), where="ipg_fused_launch")
        for e, _ in self.engines:
            e.loop_collect(sec.value)
        return sec.value

    def free(self):
        if self._p is not None and self._p.value:
            runtime().ipg_fused_free(self._p)
        self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PageRankF32:
    """PageRank with FP32 values and compensated gather sums, FP64
    diagnostics (ipg_pr_*, include/ipregel_b200.h).  Same formula and
    superstep structure as benchmarks/pagerank.c:36-66 under the
    single-broadcast version; rounds + 1 supersteps."""

    def __init__(self, graph: Graph):
        self.graph = graph
        p = ctypes.c_void_p()
        _check(runtime().ipg_pr_plan_create(graph.handle, ctypes.byref(p)), where="ipg_pr_plan_create")
        self._p = p

    def info(self) -> dict:
        cnt = np.zeros(3, np.uint64)
        edg = np.zeros(3, np.uint64)
        ch = np.zeros(1, np.uint64)
        _check(runtime().ipg_pr_plan_info(self._p, cnt.ctypes.data, edg.ctypes.data, ch.ctypes.data),
               where="ipg_pr_plan_info")
        return {"class_counts": [int(x) for x in cnt], "class_edges": [int(x) for x in edg],
                "hub_chunks": int(ch[0])}

    def run_device(self, values: DeviceArray, diag: DeviceArray, rounds=10, damping=0.85, compensated=True,
                   stream=None):
        """Enqueues a run on `stream` (a cudaStream_t as int, None = legacy
        default stream); values: V float32, diag: (rounds + 1) * 3 float64."""
        assert values.dtype == np.float32 and values.n >= self.graph.V
        assert diag.dtype == np.float64 and diag.n >= (rounds + 1) * 3
        _check(runtime().ipg_pr_run_f32(self._p, int(rounds), float(damping), int(bool(compensated)), values.ptr,
                                        diag.ptr, stream), where="ipg_pr_run_f32")

    def run(self, rounds=10, damping=0.85, compensated=True):
        """(values float32[V], diag float64[rounds + 1, 3]) with columns
        mass, dangling mass, L1 residual."""
        V = self.graph.V
        x = DeviceArray(V, np.float32)
        d = DeviceArray((rounds + 1) * 3, np.float64)
        try:
            self.run_device(x, d, rounds, damping, compensated)
            return x.to_host(), d.to_host().reshape(rounds + 1, 3)
        finally:
            x.free()
            d.free()

    def free(self):
        if self._p is not None and self._p.value:
            runtime().ipg_pr_plan_free(self._p)
        self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


PROBE_PATH = os.path.join(LIB_DIR, "libipregel_b200_probe.so")
PROBE_SYMBOLS = ("ipg_measure_gather", "ipg_probe_last_error")
_probe = None


def probe():
    """Loads the benchmark's measurement library (libipregel_b200_probe.so),
    which is not part of the runtime."""
    global _probe
    if _probe is None:
        runtime()
        if not os.path.exists(PROBE_PATH):
            raise IPregelError(f"{PROBE_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(PROBE_PATH)
        L.ipg_measure_gather.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.ipg_probe_last_error.restype = ctypes.c_char_p
        _probe = L
    return _probe


def measure_gather(table_bytes: int, row_bytes: int = 4, n: int = 1 << 28, reps: int = 5) -> dict:
    """The random-gather ceiling (ipg_measure_gather, measurement library):
    rows/s and GB/s of n scattered reads of row_bytes-byte rows from a table
    of table_bytes."""
    rows, gbs = ctypes.c_double(), ctypes.c_double()
    P = probe()
    rc = P.ipg_measure_gather(table_bytes, row_bytes, n, reps, ctypes.byref(rows), ctypes.byref(gbs))
    if rc != 0:
        raise IPregelError(f"ipg_measure_gather failed ({rc}): {P.ipg_probe_last_error().decode()}")
    return {"table_bytes": table_bytes, "row_bytes": row_bytes, "rows_per_s": rows.value, "gbs": gbs.value}


def error_f32_f64(a: DeviceArray, ref: DeviceArray, stream=None) -> dict:
    """Per-vertex error of an FP32 vector against an FP64 one, on the device."""
    n = min(a.n, ref.n)
    mx, mr, mean = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    arg = ctypes.c_uint64()
    _check(runtime().ipg_error_f32_f64(a.ptr, ref.ptr, n, ctypes.byref(mx), ctypes.byref(mr), ctypes.byref(mean),
                                       ctypes.byref(arg), stream), where="ipg_error_f32_f64")
    return {"max_abs": mx.value, "max_rel": mr.value, "mean_abs": mean.value, "argmax_abs": int(arg.value)}
