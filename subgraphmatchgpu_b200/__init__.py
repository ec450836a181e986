"""Python binding of libsme, the B200 subgraph-enumeration engine.

The engine is a drop-in for the GPU enumeration path of
guowentian/SubgraphMatchGPU: the query registry Q0..Q13 with the reference's
symmetry-breaking order (src/query/common/Query.h), the plain-BFS, LIGHT and
reuse-BFS plans (src/query/*Plan.h), the BIN CSR format
(src/graph/GraphIO.h:88-136) and the ``patternmatchgpu`` flags
(src/gpu/PatternMatchGPU.cu:17-37).  This module is a thin ctypes layer over
the C-ABI declared in include/sme.h; every call goes to the compiled library
and raises SmeError on a non-zero status.  There is no Python or CPU fallback:
without libsme.so (or without a GPU for the device entry points) calls fail.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsme.so")

# algorithms / modes (src/Meta.h:47-77)
GPU_GPSM, GPU_GPSM_REUSE, GPU_LIGHT = 4, 5, 6
IN_MEMORY_GPU, EXTERNAL_GPU = 1, 2
EXT_CACHE, EXT_UMA = 0, 1
COMPRESS_MATERIALIZE, COMPRESS_NON_MATERIALIZE, COMPRESS_NON_MATERIALIZE_OPT, COMPRESS_SPECIAL = 0, 1, 2, 3
QUERY_NAMES = {
    0: "triangle", 1: "4-cycle", 2: "diamond", 3: "4-clique", 4: "house", 5: "quad-triangle",
    6: "near-5-clique", 7: "5-clique", 8: "chordal-roof", 9: "three-triangle", 10: "solar-square",
    11: "6-clique", 12: "near-near-5-clique", 13: "triangle-in-diamond",
}

STATUS = {
    0: "OK", 1: "INVALID_ARG", 2: "BAD_FILE", 3: "OOM", 4: "TIMEOUT", 5: "CUDA", 6: "UNSUPPORTED_QUERY",
    7: "NO_DEVICE", 8: "CAPACITY", 9: "BUSY", 10: "CANCELLED",
}


class SmeError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Opts(C.Structure):
    _fields_ = [
        ("query_type", C.c_int32), ("algo", C.c_int32), ("execute_mode", C.c_int32),
        ("compress_level", C.c_int32), ("enable_ordering", C.c_int32), ("ext_variant", C.c_int32),
        ("reuse_autogen", C.c_int32), ("device", C.c_int32), ("mem_limit_bytes", C.c_uint64),
        ("root_begin", C.c_uint64), ("root_end", C.c_uint64), ("warp_granularity", C.c_int32),
        ("list_only", C.c_int32), ("root_stride", C.c_uint32), ("no_set_reuse", C.c_int32),
        ("roots", C.c_void_p), ("num_roots", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("elapsed_ms", C.c_double), ("kernel_ms", C.c_double), ("kernel_launches", C.c_uint64),
        ("batches", C.c_uint64), ("algorithmic_bytes", C.c_uint64), ("h2d_bytes", C.c_uint64),
        ("d2h_bytes", C.c_uint64), ("peak_device_bytes", C.c_uint64), ("paths_processed", C.c_uint64),
        ("device_ms", C.c_double), ("hot_launches", C.c_uint64), ("phase_ms", C.c_double * 8),
        ("reuse_hits", C.c_uint64),
    ]

    PHASES = ("compute", "materialize", "filter_compute", "compute_count", "compute_path_count", "count",
              "organize_batch", "external_load")

    def phases(self):
        return {k: self.phase_ms[i] for i, k in enumerate(self.PHASES)}


class BatchOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("autotune", C.c_int32), ("granularity", C.c_int32),
        ("block_threads", C.c_int32), ("use_graph", C.c_int32), ("reserved", C.c_int32 * 11),
    ]


class ServerOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("slots", C.c_int32), ("mem_budget_bytes", C.c_uint64),
        ("queue_capacity", C.c_int32), ("reserved", C.c_int32 * 9),
    ]


# Every entry point of include/sme.h with its ctypes signature.
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_U64 = C.c_uint64
_PU64 = C.POINTER(C.c_uint64)
SIGNATURES = {
    "sme_opts_default": (C.c_int, [C.POINTER(Opts)]),
    "sme_graph_load_bin": (C.c_int, [C.c_char_p, _PP]),
    "sme_graph_load_snap": (C.c_int, [C.c_char_p, C.c_int, _PP]),
    "sme_graph_load": (C.c_int, [C.c_char_p, C.c_int, _PP]),
    "sme_graph_from_csr": (C.c_int, [_P, _P, _U64, _U64, C.c_int, _PP]),
    "sme_graph_info": (C.c_int, [_P, _PU64, _PU64, _PU64]),
    "sme_graph_csr": (C.c_int, [_P, _PP, _PP]),
    "sme_graph_write_bin": (C.c_int, [_P, C.c_char_p]),
    "sme_graph_preprocess": (C.c_int, [_P]),
    "sme_graph_validate": (C.c_int, [_P]),
    "sme_graph_degree_order": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_void_p), C.c_void_p]),
    "sme_read_partition_file": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint32, C.c_void_p]),
    "sme_graph_load_snap_lvid": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "sme_graph_write_snap": (C.c_int, [_P, C.c_char_p]),
    "sme_graph_write_adj": (C.c_int, [_P, C.c_char_p]),
    "sme_graph_partition": (C.c_int, [_P, C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "sme_count_partitioned": (C.c_int, [_P, C.POINTER(Opts), C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64),
                                        C.c_void_p]),
    "sme_graph_is_oriented": (C.c_int32, [_P]),
    "sme_graph_to_device": (C.c_int, [_P, C.c_int]),
    "sme_graph_release_device": (C.c_int, [_P]),
    "sme_graph_device_arrays": (C.c_int, [_P, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "sme_graph_pack": (C.c_int, [_P, C.c_int, C.POINTER(C.c_uint64)]),
    "sme_graph_free": (C.c_int, [_P]),
    "sme_generate_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, _U64, _PP]),
    "sme_generate_er": (C.c_int, [_U64, C.c_double, _U64, _PP]),
    "sme_generate_ba": (C.c_int, [_U64, C.c_uint32, _U64, _PP]),
    "sme_generate_clique": (C.c_int, [_U64, _PP]),
    "sme_count": (C.c_int, [_P, C.POINTER(Opts), _PU64]),
    "sme_enumerate": (C.c_int, [_P, C.POINTER(Opts), _P, _U64, _PU64]),
    "sme_last_stats": (C.c_int, [C.POINTER(Stats)]),
    "sme_query_vertex_count": (C.c_int32, [C.c_int32]),
    "sme_plan_describe": (C.c_int, [C.c_int32, C.c_int32, C.c_char_p, _U64, _PU64]),
    "sme_batch_opts_default": (C.c_int, [C.POINTER(BatchOpts)]),
    "sme_batch_count": (C.c_int, [_P, _P, _U64, C.POINTER(BatchOpts), _P]),
    "sme_batch_prepare": (C.c_int, [_P, _P, _U64, C.POINTER(BatchOpts), _PP]),
    "sme_batch_run": (C.c_int, [_P, _P, C.POINTER(C.c_double)]),
    "sme_batch_describe": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _PU64]),
    "sme_batch_tuning": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_double)]),
    "sme_batch_free": (C.c_int, [_P]),
    "sme_count_noalloc": (C.c_int, [_P, _P, _U64, C.c_int32, _PU64]),
    "sme_server_opts_default": (C.c_int, [C.POINTER(ServerOpts)]),
    "sme_server_create": (C.c_int, [C.POINTER(ServerOpts), _PP]),
    "sme_server_add_graph": (C.c_int, [_P, _P, C.POINTER(C.c_int32)]),
    "sme_server_submit": (C.c_int, [_P, C.c_int32, _P, C.POINTER(Opts), _PU64]),
    "sme_server_poll": (C.c_int, [_P, _U64, _PU64, C.POINTER(C.c_double)]),
    "sme_server_wait": (C.c_int, [_P, _U64, _PU64, C.POINTER(C.c_double)]),
    "sme_server_stats": (C.c_int, [_P, _PU64, _PU64, _PU64]),
    "sme_server_destroy": (C.c_int, [_P]),
    "sme_last_error": (C.c_char_p, []),
    "sme_version": (C.c_char_p, []),
}

_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Loads libsme.so (built in-tree); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `make -C subgraphmatchgpu_b200/csrc` first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(st: int) -> None:
    if st != 0:
        raise SmeError(st, lib().sme_last_error().decode())


def opts(query: int = 0, algo: int = GPU_LIGHT, mode: int = IN_MEMORY_GPU, **kw) -> Opts:
    """sme_opts with the library defaults; `roots` (a sequence of vertex
    ids) makes the run an explicit root task, kept alive with the struct."""
    o = Opts()
    _check(lib().sme_opts_default(C.byref(o)))
    o.query_type, o.algo, o.execute_mode = query, algo, mode
    roots = kw.pop("roots", None)
    if roots is not None:
        r = np.ascontiguousarray(roots, dtype=np.uint32)
        o._roots = r
        o.roots = r.ctypes.data if len(r) else None
        o.num_roots = len(r)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def query_vertex_count(q: int) -> int:
    return lib().sme_query_vertex_count(q)


def plan_describe(q: int, plan_type: int) -> str:
    need = C.c_uint64(0)
    lib().sme_plan_describe(q, plan_type, None, 0, C.byref(need))
    buf = C.create_string_buffer(need.value)
    _check(lib().sme_plan_describe(q, plan_type, buf, need.value, C.byref(need)))
    return buf.value.decode()


def last_stats() -> Stats:
    s = Stats()
    _check(lib().sme_last_stats(C.byref(s)))
    return s


class Graph:
    """Owned handle of a host CSR graph (optionally resident on a device)."""

    def __init__(self, handle: int, keep=None):
        self._h = C.c_void_p(handle)
        self._keep = keep  # arrays borrowed by the library (copy=0)

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @classmethod
    def load(cls, path: str, directed: int = 0) -> "Graph":
        h = C.c_void_p()
        _check(lib().sme_graph_load(path.encode(), directed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_csr(cls, row_ptrs, cols, copy: bool = True) -> "Graph":
        rp = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
        cl = np.ascontiguousarray(cols, dtype=np.uint32)
        h = C.c_void_p()
        _check(lib().sme_graph_from_csr(rp.ctypes.data, cl.ctypes.data, len(rp) - 1, len(cl), int(copy),
                                        C.byref(h)))
        return cls(h.value, None if copy else (rp, cl))

    @classmethod
    def rmat(cls, scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed: int = 1) -> "Graph":
        h = C.c_void_p()
        _check(lib().sme_generate_rmat(scale, edge_factor, a, b, c, seed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def er(cls, n: int, avg_degree: float, seed: int = 1) -> "Graph":
        h = C.c_void_p()
        _check(lib().sme_generate_er(n, avg_degree, seed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def ba(cls, n: int, m_attach: int, seed: int = 1) -> "Graph":
        h = C.c_void_p()
        _check(lib().sme_generate_ba(n, m_attach, seed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def clique(cls, n: int) -> "Graph":
        h = C.c_void_p()
        _check(lib().sme_generate_clique(n, C.byref(h)))
        return cls(h.value)

    def info(self):
        n, m, d = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib().sme_graph_info(self._h, C.byref(n), C.byref(m), C.byref(d)))
        return n.value, m.value, d.value

    @property
    def n(self) -> int:
        return self.info()[0]

    @property
    def m(self) -> int:
        return self.info()[1]

    def csr(self):
        """Copies of (row_ptrs uint64[n+1], cols uint32[m])."""
        n, m, _ = self.info()
        rp, cl = C.c_void_p(), C.c_void_p()
        _check(lib().sme_graph_csr(self._h, C.byref(rp), C.byref(cl)))
        r = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_uint64)), shape=(n + 1,)).copy()
        c = (np.ctypeslib.as_array(C.cast(cl, C.POINTER(C.c_uint32)), shape=(m,)).copy()
             if m else np.zeros(0, np.uint32))
        return r, c

    def write_bin(self, path: str) -> None:
        _check(lib().sme_graph_write_bin(self._h, path.encode()))

    def write_snap(self, path: str) -> None:
        _check(lib().sme_graph_write_snap(self._h, path.encode()))

    def write_adj(self, path: str) -> None:
        """`path` and `path`.info (n m), the partitioner's input format."""
        _check(lib().sme_graph_write_adj(self._h, path.encode()))

    def preprocess(self) -> None:
        _check(lib().sme_graph_preprocess(self._h))

    def validate(self) -> None:
        _check(lib().sme_graph_validate(self._h))

    def degree_order(self, orient: bool = False):
        """(degree-ordered copy, new_to_old uint32[n]); `orient` keeps each
        edge once, towards the higher id (clique queries only)."""
        n = self.info()[0]
        new_to_old = np.zeros(max(n, 1), np.uint32)
        h = C.c_void_p()
        _check(lib().sme_graph_degree_order(self._h, int(orient), C.byref(h), new_to_old.ctypes.data))
        return Graph(h.value), new_to_old[:n]

    @property
    def oriented(self) -> bool:
        return bool(lib().sme_graph_is_oriented(self._h))

    def partition(self, vertex_partition, p: int) -> "Graph":
        """Subgraph induced by partition p (ascending global ids)."""
        vp = np.ascontiguousarray(vertex_partition, dtype=np.uint32)
        h = C.c_void_p()
        _check(lib().sme_graph_partition(self._h, vp.ctypes.data, p, C.byref(h)))
        return Graph(h.value)

    def count_partitioned(self, query: int, vertex_partition, partition_num: int, algo: int = GPU_LIGHT, **kw):
        """-m 0: (total, intra-partition counts per partition)."""
        vp = np.ascontiguousarray(vertex_partition, dtype=np.uint32)
        o = opts(query, algo, 0, **kw)
        total = C.c_uint64()
        intra = np.zeros(partition_num, np.uint64)
        _check(lib().sme_count_partitioned(self._h, C.byref(o), vp.ctypes.data, partition_num, C.byref(total),
                                           intra.ctypes.data))
        return total.value, intra


    def to_device(self, device: int = 0) -> None:
        _check(lib().sme_graph_to_device(self._h, device))

    def release_device(self) -> None:
        _check(lib().sme_graph_release_device(self._h))

    def device_arrays(self, device: int = 0):
        """Device addresses (row_ptrs, cols) of the resident copy on `device`."""
        rp, cl = C.c_void_p(), C.c_void_p()
        _check(lib().sme_graph_device_arrays(self._h, device, C.byref(rp), C.byref(cl)))
        return rp.value, cl.value

    def pack(self, enable: bool = True) -> int:
        """Keeps a packed copy of the lists in pinned host memory; uploads copy
        it and expand it on the device.  Returns the bytes an upload copies
        (0 after pack(False))."""
        b = C.c_uint64()
        _check(lib().sme_graph_pack(self._h, int(bool(enable)), C.byref(b)))
        return b.value

    def count(self, query: int, algo: int = GPU_LIGHT, mode: int = IN_MEMORY_GPU, **kw) -> int:
        o = opts(query, algo, mode, **kw)
        out = C.c_uint64(0)
        _check(lib().sme_count(self._h, C.byref(o), C.byref(out)))
        return out.value

    def enumerate(self, query: int, algo: int = GPU_LIGHT, cap: Optional[int] = None, **kw) -> np.ndarray:
        """All instances as a (count, k) uint32 array (pattern-vertex order)."""
        o = opts(query, algo, IN_MEMORY_GPU, **kw)
        k = query_vertex_count(query)
        if cap is None:
            cap = self.count(query, algo, **kw)
        buf = np.zeros((max(cap, 1), k), dtype=np.uint32)
        got = C.c_uint64(0)
        _check(lib().sme_enumerate(self._h, C.byref(o), buf.ctypes.data, cap, C.byref(got)))
        return buf[: got.value]

    def close(self) -> None:
        if self._h and self._h.value:
            lib().sme_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """Batched form: many small (graph, query) pairs, one persistent launch
    captured in a CUDA graph, group size and block shape autotuned."""

    def __init__(self, graphs: Sequence[Graph], queries: Sequence[int], autotune: bool = True,
                 use_graph: bool = True, device: int = 0, granularity: int = 0, block_threads: int = 0):
        o = BatchOpts()
        _check(lib().sme_batch_opts_default(C.byref(o)))
        o.autotune, o.use_graph, o.device = int(autotune), int(use_graph), device
        o.granularity, o.block_threads = granularity, block_threads
        self._graphs = list(graphs)
        hs = (C.c_void_p * len(graphs))(*[g.handle.value for g in graphs])
        qs = np.ascontiguousarray(queries, dtype=np.int32)
        self._h = C.c_void_p()
        _check(lib().sme_batch_prepare(hs, qs.ctypes.data, len(graphs), C.byref(o), C.byref(self._h)))
        self.num = len(graphs)

    def run(self):
        counts = np.zeros(self.num, dtype=np.uint64)
        ms = C.c_double(0)
        _check(lib().sme_batch_run(self._h, counts.ctypes.data, C.byref(ms)))
        return counts, ms.value

    def describe(self):
        g, b, n = C.c_int32(), C.c_int32(), C.c_uint64()
        _check(lib().sme_batch_describe(self._h, C.byref(g), C.byref(b), C.byref(n)))
        c, ms = C.c_int32(), C.c_double()
        _check(lib().sme_batch_tuning(self._h, None, None, C.byref(c), C.byref(ms)))
        return {"group_threads": g.value, "block_threads": b.value, "work_items": n.value,
                "items_per_fetch": c.value, "tuned_ms": ms.value}

    def close(self):
        if self._h and self._h.value:
            lib().sme_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Served form: resident graphs, admission by estimated frontier memory,
    concurrent requests across slots (continuous batching)."""

    def __init__(self, slots: int = 4, mem_budget_bytes: int = 0, device: int = 0, queue_capacity: int = 1 << 16):
        o = ServerOpts()
        _check(lib().sme_server_opts_default(C.byref(o)))
        o.slots, o.mem_budget_bytes, o.device, o.queue_capacity = slots, mem_budget_bytes, device, queue_capacity
        self._h = C.c_void_p()
        _check(lib().sme_server_create(C.byref(o), C.byref(self._h)))
        self._keep = []

    def add_graph(self, g: Graph) -> int:
        gid = C.c_int32()
        _check(lib().sme_server_add_graph(self._h, g.handle, C.byref(gid)))
        self._keep.append(g)
        return gid.value

    def submit(self, query: int, gid: int = -1, attached: Optional[Graph] = None, algo: int = GPU_LIGHT,
               **kw) -> int:
        o = opts(query, algo, IN_MEMORY_GPU, **kw)
        rid = C.c_uint64()
        if attached is not None:
            self._keep.append(attached)
        _check(lib().sme_server_submit(self._h, gid, attached.handle if attached is not None else None,
                                       C.byref(o), C.byref(rid)))
        return rid.value

    def poll(self, rid: int):
        c, lat = C.c_uint64(), C.c_double()
        st = lib().sme_server_poll(self._h, rid, C.byref(c), C.byref(lat))
        if st == 9:
            return None
        _check(st)
        return c.value, lat.value

    def wait(self, rid: int):
        c, lat = C.c_uint64(), C.c_double()
        _check(lib().sme_server_wait(self._h, rid, C.byref(c), C.byref(lat)))
        return c.value, lat.value

    def stats(self):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib().sme_server_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"completed": a.value, "max_inflight": b.value, "rejected": c.value}

    def close(self):
        if self._h and self._h.value:
            lib().sme_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = [
    "BatchPlan", "Server",
    "Graph", "SmeError", "Opts", "Stats", "lib", "opts", "plan_describe", "last_stats", "query_vertex_count",
    "read_partition_file",
    "GPU_GPSM", "GPU_GPSM_REUSE", "GPU_LIGHT", "IN_MEMORY_GPU", "EXTERNAL_GPU", "SIGNATURES", "QUERY_NAMES",
]


def read_partition_file(path: str, n: int, partition_num: int) -> np.ndarray:
    """GraphIO::ReadPartitionFile: uint32 partition id per vertex."""
    out = np.zeros(max(n, 1), np.uint32)
    _check(lib().sme_read_partition_file(path.encode(), n, partition_num, out.ctypes.data))
    return out[:n]
