"""gem_filter_static: the candidate filter for callers that cannot allocate
device memory (code inside another framework's allocator or memory pool, or
a service whose memory is reserved up front).  The test owns every device buffer (torch
allocates them); the entry point itself allocates nothing and keeps its
scratch in a fixed device array.  Its output must equal gem_filter's (the
allocating entry point) bit for bit, on two calls in a row — the second call
reuses the scratch the first one left behind.  This file sorts last so a
run that stops at the first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

import gem_b200 as gem

pytestmark = pytest.mark.gpu


def _dev(arr, torch, dtype):
    return torch.from_numpy(np.array(arr, copy=True).view(dtype)).cuda()


def test_filter_static_matches_gem_filter():
    import torch
    g = gem.HostGraph.rmat(13, 8, seed=0x5A11).set_labels(5, 0.5, seed=0x5A12)
    off, nbr, lab = g.arrays()
    d_off = _dev(off.astype(np.uint64), torch, np.int64)
    d_nbr = _dev(nbr.astype(np.uint32), torch, np.int32)
    d_lab = _dev(lab.astype(np.uint32), torch, np.int32)
    qs = gem.gen_queries(g, 6, gem.ANY, 2, seed=0x5A13) + gem.gen_queries(g, 4, gem.DENSE, 2, seed=0x5A14)
    ts = [i % 3 for i in range(len(qs))]  # thresholds 0, 1, 2
    with gem.Context(time_cap_ms=20000) as ctx:
        ctx.load_graph(g)
        expected = [ctx.filter(q, threshold=t) for q, t in zip(qs, ts)]
    L = gem.lib()
    for call in range(2):  # two calls in a row share the static scratch
        for q, t, exp in zip(qs, ts, expected):
            total = sum(len(x) for x in exp)
            d_cand = torch.full((total + 64,), -1, dtype=torch.int32, device="cuda")
            counts = np.zeros(q.nv, np.uint32)
            qc = q._c()
            torch.cuda.synchronize()
            st = L.gem_filter_static(C.c_void_p(d_off.data_ptr()), C.c_void_p(d_nbr.data_ptr()),
                                     C.c_void_p(d_lab.data_ptr()), g.nv, C.byref(qc), t,
                                     counts.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_void_p(d_cand.data_ptr()),
                                     total + 64, None)
            assert st == 0, (call, gem.STATUS.get(st, st))
            cand = d_cand.cpu().numpy().view(np.uint32)
            at = 0
            for u in range(q.nv):
                assert counts[u] == len(exp[u]), (call, u)
                assert np.array_equal(cand[at:at + counts[u]], exp[u]), (call, u)
                at += int(counts[u])
            assert np.all(cand[at:] == 0xFFFFFFFF)  # nothing written past the lists


def test_filter_static_rejects_oversized_graph():
    q = gem.Query([0, 1], [(0, 1)])
    qc = q._c()
    counts = np.zeros(2, np.uint32)
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = gem.lib().gem_filter_static(one, one, one, 8_000_001, C.byref(qc), 0,
                                     counts.ctypes.data_as(C.POINTER(C.c_uint32)), one, 0, None)
    assert gem.STATUS[st] == "ERR_LIMIT"


def test_filter_static_reports_malformed_graph():
    """A neighbour id beyond the vertex count is skipped on the device (never
    used as an index) and the call returns GEM_ERR_ARG; the next call on a
    well-formed graph is exact again."""
    import torch
    g = gem.HostGraph.rmat(10, 8, seed=0x5A21).set_labels(3, 0.0, seed=0x5A22)
    off, nbr, lab = g.arrays()
    v = int(np.argmax(np.diff(off.astype(np.int64))))  # a vertex with neighbours
    q = gem.Query([int(lab[v]), int(lab[nbr[off[v]]])], [(0, 1)])
    bad_nbr = nbr.astype(np.uint32).copy()
    bad_nbr[off[v]] = g.nv + 1000
    d_off = _dev(off.astype(np.uint64), torch, np.int64)
    d_lab = _dev(lab.astype(np.uint32), torch, np.int32)
    L = gem.lib()
    qc = q._c()
    for arr, want in ((bad_nbr, "ERR_ARG"), (nbr.astype(np.uint32), "OK")):
        d_nbr = _dev(arr, torch, np.int32)
        d_cand = torch.full((2 * g.nv,), -1, dtype=torch.int32, device="cuda")
        counts = np.zeros(q.nv, np.uint32)
        torch.cuda.synchronize()
        st = L.gem_filter_static(C.c_void_p(d_off.data_ptr()), C.c_void_p(d_nbr.data_ptr()),
                                 C.c_void_p(d_lab.data_ptr()), g.nv, C.byref(qc), 0,
                                 counts.ctypes.data_as(C.POINTER(C.c_uint32)), C.c_void_p(d_cand.data_ptr()),
                                 2 * g.nv, None)
        assert gem.STATUS[st] == want


def test_filter_static_rejects_null_adjacency():
    q = gem.Query([0, 1], [(0, 1)])
    qc = q._c()
    counts = np.zeros(2, np.uint32)
    one = C.c_void_p(1)  # never dereferenced: the argument check comes first
    st = gem.lib().gem_filter_static(one, None, one, 16, C.byref(qc), 0,
                                     counts.ctypes.data_as(C.POINTER(C.c_uint32)), one, 0, None)
    assert gem.STATUS[st] == "ERR_ARG"
