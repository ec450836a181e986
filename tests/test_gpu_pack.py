"""Packed uploads (sme_graph_pack): the device expansion of the packed lists
against the host CSR, word for word, and counts through packed uploads
against the reference's golden counts.  Also the hub bitmaps, built in shared
memory, with every vertex a hub."""
import numpy as np
import pytest

import subgraphmatchgpu_b200 as sme
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu

GOLDEN = ("ba_n600_m4", "er_n600_d8", "rmat_s10_ef8", "rmat_s12_ef8", "k20")


def device_csr(g, device=0):
    """The resident copy's arrays, read back through the CUDA runtime."""
    from cuda.bindings import runtime as rt
    rp_ptr, cl_ptr = g.device_arrays(device)
    rp = np.empty(g.n + 1, np.uint64)
    cl = np.empty(max(g.m, 1), np.uint32)
    for host, dev in ((rp, rp_ptr), (cl, cl_ptr)):
        err, = rt.cudaMemcpy(host.ctypes.data, dev, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert int(err) == 0, err
    return rp, cl[:g.m]


def edge_case_graph(seed):
    """Lists at every block and segment boundary (0, 1, 31-33, 1023-1025,
    2047-2049 elements), sorted with small and large gaps, unsorted, with
    repeats and with the largest vertex id; the packing is modular, so any
    list must come back as it was."""
    rng = np.random.default_rng(seed)
    n = 3000
    lens = [0, 1, 31, 32, 33, 63, 64, 65, 1023, 1024, 1025, 2047, 2048, 2049]
    rows, cols = [0], []
    for u in range(n):
        d = lens[u % len(lens)] if u < 4 * len(lens) else int(rng.integers(0, 90))
        kind = u % 4
        if kind == 0:
            lst = np.sort(rng.choice(n, size=min(d, n), replace=False))
        elif kind == 1:
            lst = np.sort(rng.integers(0, n, size=d))  # repeats
        elif kind == 2:
            lst = rng.integers(0, n, size=d)  # unsorted
        else:
            lst = np.sort(rng.integers(0, n, size=d))
            if d:
                lst[-1] = n - 1
        cols.extend(int(x) for x in lst)
        rows.append(len(cols))
    return sme.Graph.from_csr(np.array(rows, np.uint64), np.array(cols, np.uint32))


@pytest.mark.parametrize("name", GOLDEN)
def test_packed_upload_expands_to_the_host_csr(name):
    g = sme.Graph.load(golden_graph_path(name))
    plain = (g.n + 1) * 8 + g.m * 4
    b = g.pack()
    assert 0 < b < plain
    g.to_device(0)
    rp, cl = device_csr(g)
    hrp, hcl = g.csr()
    assert np.array_equal(rp, hrp)
    assert np.array_equal(cl, hcl)


@pytest.mark.parametrize("seed", [1, 2])
def test_packed_upload_of_boundary_lists(seed):
    g = edge_case_graph(seed)
    g.pack()
    g.to_device(0)
    rp, cl = device_csr(g)
    hrp, hcl = g.csr()
    assert np.array_equal(rp, hrp)
    assert np.array_equal(cl, hcl)


def test_packed_upload_of_rmat_s16_lists():
    # lists of up to a few thousand elements: many segments per list
    g = sme.Graph.rmat(16, 16, seed=16)
    b = g.pack()
    assert b < 0.6 * ((g.n + 1) * 8 + g.m * 4)
    g.to_device(0)
    rp, cl = device_csr(g)
    hrp, hcl = g.csr()
    assert np.array_equal(rp, hrp)
    assert np.array_equal(cl, hcl)


@pytest.mark.parametrize("name", GOLDEN)
def test_counts_through_packed_per_call_uploads(golden, name):
    # not resident: every call uploads the packed lists into its arena
    g = sme.Graph.load(golden_graph_path(name))
    b = g.pack()
    want = golden[name]["counts"]
    for q in (0, 1, 3, 4, 7):
        for algo in (sme.GPU_LIGHT, sme.GPU_GPSM):
            assert g.count(q, algo) == want[str(q)], (name, q, algo)
            s = sme.last_stats()
            assert b <= s.h2d_bytes < b + 4 * g.n + 4096, (s.h2d_bytes, b)


def test_repacking_follows_the_lists_and_unpacking_restores_the_plain_upload(golden):
    g = sme.Graph.load(golden_graph_path("rmat_s12_ef8"))
    want = golden["rmat_s12_ef8"]["counts"]
    plain = (g.n + 1) * 8 + g.m * 4
    g.pack()
    g.pack()
    assert g.count(3) == want["3"]
    assert g.pack(False) == 0
    assert g.count(3) == want["3"]
    assert sme.last_stats().h2d_bytes >= plain


def test_every_vertex_a_hub(golden, monkeypatch):
    # SME_HUB_MIN_DEGREE=1: every vertex with a list gets a bitmap (built in
    # shared memory, one CTA per hub); counts unchanged
    monkeypatch.setenv("SME_HUB_MIN_DEGREE", "1")
    for name in ("ba_n600_m4", "rmat_s10_ef8"):
        g = sme.Graph.load(golden_graph_path(name))
        g.pack()
        want = golden[name]["counts"]
        for q in (0, 1, 2, 3, 4, 9):
            assert g.count(q) == want[str(q)], (name, q)
        g.to_device(0)
        for q in (0, 3, 4):
            assert g.count(q, sme.GPU_GPSM_REUSE) == want[str(q)], (name, q)


def test_per_call_packed_upload_in_ranges_counts_as_resident():
    # an s18 graph packs to more than 8 MB, so a per-call upload is cut into
    # ranges whose copy overlaps the expansion and the hub bitmaps
    g = sme.Graph.rmat(18, 16, seed=18)
    assert g.pack() >= 8 << 20
    got = {q: g.count(q, root_begin=q, root_stride=32) for q in (0, 1, 2, 3, 4)}
    got[0, "all"] = g.count(0)
    g.pack(False)
    g.to_device(0)
    want = {q: g.count(q, root_begin=q, root_stride=32) for q in (0, 1, 2, 3, 4)}
    want[0, "all"] = g.count(0)
    assert got == want
