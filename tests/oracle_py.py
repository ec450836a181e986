"""ctypes loader of the CPU oracle (oracle/liboracle.so) -- test infrastructure.

Used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
LIB = os.path.join(ROOT, "oracle", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
        L = C.CDLL(LIB)
        L.oracle_wcoj.restype = C.c_uint64
        L.oracle_wcoj.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                  C.c_int, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]
        L.oracle_query_size.restype = C.c_int
        L.oracle_query_size.argtypes = [C.c_int]
        L.oracle_wcoj_sample.restype = C.c_uint64
        L.oracle_wcoj_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_void_p,
                                         C.c_uint64, C.c_int, C.c_double, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_double)]
        L.oracle_wcoj_strided.restype = C.c_uint64
        L.oracle_wcoj_strided.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_uint64,
                                          C.c_uint64, C.c_int]
        L.oracle_write_edge_text.restype = C.c_int
        L.oracle_write_edge_text.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_char_p]
        _lib = L
    return _lib


def count(row_ptrs, cols, q, ordering=True, root_begin=0, root_end=0, threads=0) -> int:
    rp = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
    cl = np.ascontiguousarray(cols, dtype=np.uint32)
    return int(lib().oracle_wcoj(rp.ctypes.data, cl.ctypes.data if len(cl) else None, len(rp) - 1, q,
                                 int(ordering), root_begin, root_end, threads, None, 0, None))


def count_strided(row_ptrs, cols, q, stride, offset=0, threads=0, ordering=True) -> int:
    rp = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
    cl = np.ascontiguousarray(cols, dtype=np.uint32)
    return int(lib().oracle_wcoj_strided(rp.ctypes.data, cl.ctypes.data if len(cl) else None, len(rp) - 1, q,
                                         int(ordering), stride, offset, threads))


def count_sample(row_ptrs, cols, q, roots, budget_s, threads=0, ordering=True):
    """Time-bounded sample: (instances of completed roots, completed roots,
    seconds); roots cut short by the deadline are discarded."""
    rp = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
    cl = np.ascontiguousarray(cols, dtype=np.uint32)
    rt = np.ascontiguousarray(roots, dtype=np.uint32)
    done, el = C.c_uint64(0), C.c_double(0)
    inst = lib().oracle_wcoj_sample(rp.ctypes.data, cl.ctypes.data if len(cl) else None, len(rp) - 1, q,
                                    int(ordering), rt.ctypes.data, len(rt), threads, budget_s, C.byref(done),
                                    C.byref(el))
    return int(inst), int(done.value), float(el.value)


def count_roots(row_ptrs, cols, q, roots, threads=0, ordering=True) -> int:
    """Instances rooted at exactly the vertices of `roots` (an explicit root
    task; a root listed twice counts twice)."""
    inst, done, _ = count_sample(row_ptrs, cols, q, roots, 1e12, threads, ordering)
    assert done == len(roots)
    return inst


def preprocess_csr(row_ptrs, cols):
    """PreprocessGraph::Preprocess (src/preprocess/PreprocessGraph.h:13-95) in
    numpy: drop self loops and repeated neighbours of sorted lists, then the
    vertices left without edges, relabelling the rest densely in id order."""
    rp = np.asarray(row_ptrs, np.uint64).astype(np.int64)
    cl = np.asarray(cols, np.uint32)
    n = len(rp) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    keep = cl.astype(np.int64) != src
    keep[1:] &= ~((cl[1:] == cl[:-1]) & (src[1:] == src[:-1]))
    src, dst = src[keep], cl[keep].astype(np.int64)
    deg = np.bincount(src, minlength=n)
    new_id = np.cumsum(deg > 0) - 1
    nrp = np.zeros(int((deg > 0).sum()) + 1, np.uint64)
    nrp[1:] = np.cumsum(deg[deg > 0])
    return nrp, new_id[dst].astype(np.uint32)


def write_edge_text(u, v, path) -> None:
    """SNAP text edge list ("u v" per line) for the reference's tools."""
    uu = np.ascontiguousarray(u, dtype=np.uint32)
    vv = np.ascontiguousarray(v, dtype=np.uint32)
    if lib().oracle_write_edge_text(uu.ctypes.data, vv.ctypes.data, len(uu), path.encode()) != 0:
        raise OSError(f"cannot write {path}")


def enumerate_sorted(row_ptrs, cols, q, ordering=True) -> np.ndarray:
    rp = np.ascontiguousarray(row_ptrs, dtype=np.uint64)
    cl = np.ascontiguousarray(cols, dtype=np.uint32)
    k = lib().oracle_query_size(q)
    n = count(rp, cl, q, ordering)
    buf = np.zeros((max(n, 1), k), dtype=np.uint32)
    got = C.c_uint64(0)
    lib().oracle_wcoj(rp.ctypes.data, cl.ctypes.data if len(cl) else None, len(rp) - 1, q, int(ordering), 0, 0,
                      0, buf.ctypes.data, n, C.byref(got))
    out = buf[: got.value]
    return sort_rows(out)


def sort_rows(a: np.ndarray) -> np.ndarray:
    if len(a) == 0:
        return a
    idx = np.lexsort(tuple(a[:, j] for j in reversed(range(a.shape[1]))))
    return a[idx]


def read_bin(path):
    """BIN CSR reader for fixtures (4 x size_t header, row_ptrs, cols)."""
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw[:32], dtype=np.uint64)
    n, m = int(hdr[2]), int(hdr[3])
    rp = np.frombuffer(raw[32:32 + 8 * (n + 1)], dtype=np.uint64).copy()
    cl = np.frombuffer(raw[32 + 8 * (n + 1):32 + 8 * (n + 1) + 4 * m], dtype=np.uint32).copy()
    return rp, cl
