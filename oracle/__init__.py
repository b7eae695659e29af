"""CPU oracle — TEST INFRASTRUCTURE ONLY.

ctypes binding to oracle/_build/liboracle.so (built from oracle/oracle.c by
gem_b200.build / __graft_entry__.build).  Only the test suite, the smoke
check and the CPU-baseline leg of bench.py may import this module; libgem
never uses it.  See oracle/oracle.c for the reference semantics it restates.
"""
import ctypes as C
import os

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_DIR, "_build", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"oracle not built at {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        u32p, u64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
        L.oracle_emb_hash.argtypes = [u32p, C.c_uint32]
        L.oracle_emb_hash.restype = C.c_uint64
        L.oracle_filter.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32,
                                    u32p, u32p, C.c_uint64]
        L.oracle_edge_table.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, u64p, u32p,
                                        C.c_uint64]
        L.oracle_edge_table.restype = C.c_int64
        L.oracle_filter_mt.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, u32p,
                                       C.c_uint32, u32p, u32p, C.c_uint64, C.c_int]
        L.oracle_edge_table_mt.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, u64p, u32p,
                                           C.c_uint64, C.c_int]
        L.oracle_edge_table_mt.restype = C.c_int64
        L.oracle_count.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, u32p, C.c_int,
                                   C.c_int, C.c_uint64, u64p, u64p, u64p]
        L.oracle_brute.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, u32p, C.c_uint32, u32p, u64p, u64p]
        L.oracle_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64, u64p,
                                  C.POINTER(u32p), u64p]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_free.restype = None
        L.oracle_set_labels.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, u32p]
        L.oracle_gen_queries.argtypes = [C.c_uint32, u64p, u32p, u32p, C.c_uint32, C.c_int, C.c_uint32, C.c_uint64,
                                         C.c_uint32, u32p, u32p, u32p]
        _lib = L
    return _lib


def _p32(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _graph(g):
    """Accepts (offsets, nbrs, labels) numpy arrays or any object with .arrays()."""
    off, nbr, lab = g.arrays() if hasattr(g, "arrays") else g
    off = np.ascontiguousarray(off, dtype=np.uint64)
    nbr = np.ascontiguousarray(nbr, dtype=np.uint32)
    if nbr.size == 0:
        nbr = np.zeros(1, np.uint32)
    lab = np.ascontiguousarray(lab, dtype=np.uint32)
    return off, nbr, lab


def _query(q):
    lab = np.ascontiguousarray(q.labels, dtype=np.uint32)
    edg = np.ascontiguousarray(q.edges, dtype=np.uint32).reshape(-1)
    if edg.size == 0:
        edg = np.zeros(2, np.uint32)
    return lab, edg, int(q.labels.shape[0]), int(q.edges.shape[0])


def emb_hash(f):
    f = np.ascontiguousarray(f, dtype=np.uint32)
    return int(lib().oracle_emb_hash(_p32(f), len(f)))


def count(g, q, threads=0, want_hash=True, work_cap=0):
    """(count, hash, complete) by backtracking; work_cap bounds scanned arcs."""
    off, nbr, lab = _graph(g)
    ql, qe, qn, qm = _query(q)
    c, h, n = C.c_uint64(), C.c_uint64(), C.c_uint64()
    r = lib().oracle_count(len(lab), _p64(off), _p32(nbr), _p32(lab), qn, _p32(ql), qm, _p32(qe), threads,
                           1 if want_hash else 0, work_cap, C.byref(c), C.byref(h), C.byref(n))
    if r < 0:
        raise ValueError("oracle_count rejected the query")
    return int(c.value), int(h.value), r == 0


def brute(g, q):
    off, nbr, lab = _graph(g)
    ql, qe, qn, qm = _query(q)
    c, h = C.c_uint64(), C.c_uint64()
    r = lib().oracle_brute(len(lab), _p64(off), _p32(nbr), _p32(lab), qn, _p32(ql), qm, _p32(qe), C.byref(c),
                           C.byref(h))
    if r != 0:
        raise ValueError("brute force supports nv <= 64 data vertices and <= 8 query vertices")
    return int(c.value), int(h.value)


def filter(g, q, threshold=0):
    off, nbr, lab = _graph(g)
    ql, qe, qn, qm = _query(q)
    counts = np.zeros(qn, np.uint32)
    cap = qn * len(lab)
    cand = np.zeros(max(cap, 1), np.uint32)
    r = lib().oracle_filter(len(lab), _p64(off), _p32(nbr), _p32(lab), qn, _p32(ql), qm, _p32(qe), threshold,
                            _p32(counts), _p32(cand), cap)
    assert r == 0
    out, at = [], 0
    for u in range(qn):
        out.append(cand[at:at + int(counts[u])].copy())
        at += int(counts[u])
    return out


def filter_mt(g, q, threshold=0, threads=0):
    """filter() on threads (0: the reference's out-of-core worker count, min(16, all))."""
    off, nbr, lab = _graph(g)
    ql, qe, qn, qm = _query(q)
    counts = np.zeros(qn, np.uint32)
    cap = qn * len(lab)
    cand = np.zeros(max(cap, 1), np.uint32)
    r = lib().oracle_filter_mt(len(lab), _p64(off), _p32(nbr), _p32(lab), qn, _p32(ql), qm, _p32(qe), threshold,
                               _p32(counts), _p32(cand), cap, threads)
    assert r == 0
    out, at = [], 0
    for u in range(qn):
        out.append(cand[at:at + int(counts[u])].copy())
        at += int(counts[u])
    return out


def edge_table_mt(g, cu, cw, threads=0):
    """edge_table() on threads (0: the reference's out-of-core worker count, min(4, all))."""
    off, nbr, lab = _graph(g)
    cu = np.ascontiguousarray(cu, dtype=np.uint32)
    cw = np.ascontiguousarray(cw, dtype=np.uint32)
    offsets = np.zeros(len(cu) + 1, np.uint64)
    cap = int((off[cu.astype(np.int64) + 1] - off[cu.astype(np.int64)]).sum()) + 1 if len(cu) else 1
    vals = np.zeros(cap, np.uint32)
    r = lib().oracle_edge_table_mt(len(lab), _p64(off), _p32(nbr),
                                   _p32(cu if cu.size else np.zeros(1, np.uint32)), len(cu),
                                   _p32(cw if cw.size else np.zeros(1, np.uint32)), len(cw), _p64(offsets),
                                   _p32(vals), cap, threads)
    assert r >= 0
    return offsets, vals[:r].copy()


def edge_table(g, cu, cw):
    off, nbr, lab = _graph(g)
    cu = np.ascontiguousarray(cu, dtype=np.uint32)
    cw = np.ascontiguousarray(cw, dtype=np.uint32)
    offsets = np.zeros(len(cu) + 1, np.uint64)
    cap = int(sum(int(off[v + 1] - off[v]) for v in cu)) + 1
    vals = np.zeros(cap, np.uint32)
    r = lib().oracle_edge_table(len(lab), _p64(off), _p32(nbr), _p32(cu if cu.size else np.zeros(1, np.uint32)),
                                len(cu), _p32(cw if cw.size else np.zeros(1, np.uint32)), len(cw), _p64(offsets),
                                _p32(vals), cap)
    assert r >= 0
    return offsets, vals[:r].copy()


class Graph:
    """A data graph as plain numpy CSR arrays (offsets u64[nv+1], nbrs u32[arcs], labels u32[nv]),
    accepted wherever the functions above take a graph."""

    def __init__(self, off, nbr, lab):
        self.off, self.nbr, self.lab = off, nbr, lab

    @property
    def nv(self):
        return int(self.lab.shape[0])

    def arrays(self):
        return self.off, self.nbr, self.lab


class Query:
    """A query: labels u32[nv] and undirected edges u32[ne, 2]."""

    def __init__(self, labels, edges):
        self.labels = np.ascontiguousarray(labels, dtype=np.uint32)
        self.edges = np.ascontiguousarray(edges, dtype=np.uint32).reshape(-1, 2)

    @property
    def nv(self):
        return int(self.labels.shape[0])

    @property
    def ne(self):
        return int(self.edges.shape[0])


def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=None):
    """Seeded R-MAT graph (oracle_rmat) with all labels 0; equal to gem_hgraph_rmat's."""
    seed = (0x47454D00 + scale) if seed is None else seed
    nv = 1 << scale
    off = np.zeros(nv + 1, np.uint64)
    pn = C.POINTER(C.c_uint32)()
    na = C.c_uint64()
    if lib().oracle_rmat(scale, edge_factor, a, b, c, seed, _p64(off), C.byref(pn), C.byref(na)) != 0:
        raise MemoryError("oracle_rmat failed")
    try:
        nbr = np.ctypeslib.as_array(pn, shape=(max(na.value, 1),))[:na.value].copy()
    finally:
        lib().oracle_free(pn)
    return Graph(off, nbr, np.zeros(nv, np.uint32))


def set_labels(g, nlabels, zipf_s=0.0, seed=0x47454D4C):
    """Seeded labels (oracle_set_labels), in place; equal to gem_hgraph_set_labels's."""
    lab = np.zeros(g.nv, np.uint32)
    if lib().oracle_set_labels(g.nv, nlabels, zipf_s, seed, _p32(lab)) != 0:
        raise ValueError("oracle_set_labels rejected its arguments")
    g.lab = lab
    return g


def gen_queries(g, k, density=0, count=1, seed=0x51000, max_e=496):
    """Seeded random-walk queries (oracle_gen_queries); equal to gem_gen_queries's."""
    off, nbr, lab = _graph(g)
    ne = np.zeros(count, np.uint32)
    ql = np.zeros(max(count * k, 1), np.uint32)
    qe = np.zeros(max(count * 2 * max_e, 1), np.uint32)
    r = lib().oracle_gen_queries(len(lab), _p64(off), _p32(nbr), _p32(lab), k, density, count, seed, max_e,
                                 _p32(ne), _p32(ql), _p32(qe))
    if r != 0:
        raise ValueError(f"oracle_gen_queries failed ({r})")
    return [Query(ql[i * k:(i + 1) * k].copy(),
                  qe[i * 2 * max_e: i * 2 * max_e + 2 * int(ne[i])].reshape(-1, 2).copy()) for i in range(count)]
