"""sme_count_noalloc: the allocation-free entry point.

Some callers cannot call cudaMalloc — for example code that runs inside a
framework whose caching allocator has already reserved the GPU's memory, or a
latency-critical path that cannot pay for an allocation and the
synchronisation it brings.  They hand the library a CSR that already lives in
device memory, and the library counts with nothing but its own fixed 16 MiB
device array as scratch.  This file checks, through the C-ABI, that two calls
in a row return exactly the counts of the regular entry point (sme_count), and
that inputs beyond the stated limit are refused with a clear error.  It is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

import subgraphmatchgpu_b200 as sme
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu

COUNT_LIMIT = 300_000_000  # keeps this file to seconds


def device_csr(g):
    """The test (the caller) owns the device copy of the CSR."""
    import torch
    rp, cl = g.csr()
    d_rp = torch.from_numpy(rp.view(np.int64).copy()).cuda()
    d_cl = torch.from_numpy(cl.view(np.int32).copy() if len(cl) else np.zeros(1, np.int32)).cuda()
    torch.cuda.synchronize()
    return d_rp, d_cl, len(rp) - 1


def count_noalloc(d_rp, d_cl, n, q):
    out = C.c_uint64(0)
    st = sme.lib().sme_count_noalloc(d_rp.data_ptr(), d_cl.data_ptr(), n, q, C.byref(out))
    return st, out.value


@pytest.mark.parametrize("name", ["er_n64_d12", "ba_n600_m4", "k12", "rmat_s10_ef8"])
def test_noalloc_matches_regular_entry_point_twice(name, golden):
    g = sme.Graph.load(golden_graph_path(name))
    d_rp, d_cl, n = device_csr(g)
    checked = 0
    for q in range(14):
        want_ref = golden[name]["counts"].get(str(q))
        if want_ref is not None and want_ref > COUNT_LIMIT:
            continue
        want = g.count(q)  # the existing entry point
        if want_ref is not None:
            assert want == want_ref, (name, q, want, want_ref)
        for _ in range(2):  # two calls in a row share (and reuse) the scratch
            st, got = count_noalloc(d_rp, d_cl, n, q)
            assert st == 0, sme.lib().sme_last_error().decode()
            assert got == want, (name, q, got, want)
        checked += 1
    assert checked >= 8


def test_noalloc_rejects_sizes_beyond_the_limit():
    # a star whose centre has degree 40000 > 32768
    leaves = 40000
    rp = np.zeros(leaves + 2, np.uint64)
    rp[1] = leaves
    rp[2:] = leaves + np.arange(1, leaves + 1, dtype=np.uint64)
    cl = np.concatenate([np.arange(1, leaves + 1, dtype=np.uint32), np.zeros(leaves, np.uint32)])
    g = sme.Graph.from_csr(rp, cl)
    d_rp, d_cl, n = device_csr(g)
    st, _ = count_noalloc(d_rp, d_cl, n, 0)
    assert st == 8  # SME_ERR_CAPACITY
    assert "32768" in sme.lib().sme_last_error().decode()
    st, _ = count_noalloc(d_rp, d_cl, n, 14)
    assert st == 6  # unknown query
    # the entry point stays usable afterwards
    g2 = sme.Graph.clique(6)
    d_rp2, d_cl2, n2 = device_csr(g2)
    assert count_noalloc(d_rp2, d_cl2, n2, 3) == (0, 15)


def test_noalloc_rejects_lists_that_break_the_input_contract():
    # K6 with one list made unsorted, one with a self loop, one with a
    # duplicate neighbour: the sorted-list searches would count wrongly, so
    # each is refused with INVALID_ARG before any enumeration
    rp, cl = sme.Graph.clique(6).csr()
    bad = []
    c = cl.copy()
    c[0], c[1] = c[1], c[0]
    bad.append(c)
    c = cl.copy()
    c[int(rp[2])] = 2  # vertex 2 lists itself
    bad.append(c)
    c = cl.copy()
    c[int(rp[3]) + 1] = c[int(rp[3])]  # duplicate neighbour in vertex 3's list
    bad.append(c)
    for c in bad:
        import torch
        d_rp = torch.from_numpy(rp.view(np.int64).copy()).cuda()
        d_cl = torch.from_numpy(c.view(np.int32).copy()).cuda()
        torch.cuda.synchronize()
        st, _ = count_noalloc(d_rp, d_cl, len(rp) - 1, 0)
        assert st == 1, sme.lib().sme_last_error().decode()
        assert "strictly increasing" in sme.lib().sme_last_error().decode()
    d_rp, d_cl, n = device_csr(sme.Graph.clique(6))
    assert count_noalloc(d_rp, d_cl, n, 0) == (0, 20)
