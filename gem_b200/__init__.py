"""gem_b200 — Python view of libgem, a B200-native edge-centric subgraph matcher.

Everything here is a thin ctypes layer over the C-ABI declared in
include/gem.h; the work happens in libgem.so (C++ host code and sm_100a CUDA
kernels).  There is no CPU fallback: if libgem.so is missing or no CUDA device
is present, device calls raise.

Typical use::

    import gem_b200 as gem
    g = gem.HostGraph.rmat(scale=16, edge_factor=8, seed=1).set_labels(8)
    qs = gem.gen_queries(g, k=4, density=gem.SPARSE, count=10, seed=7)
    ctx = gem.Context()
    ctx.load_graph(g)
    res = ctx.run(qs[0])            # exact embedding count (u64)

The reference's driver surface is `GEM -q <query> -d <data> -t 0`
(in-core/src/main.cu:23-275); `gem_b200/bin/gem` is the drop-in CLI and this
module mirrors its phases (filter, hash index, edge tables, join) for tests
and tools.
"""
import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libgem.so")

ANY, SPARSE, DENSE = 0, 1, 2
MODE_COUNT, MODE_HASH, MODE_ENUMERATE = 0, 1, 2
IDX_AUTO, IDX_RANK, IDX_CUCKOO = 0, 1, 2
MAX_QV, MAX_QE = 32, 496

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_OOM", 3: "ERR_LIMIT", 4: "ERR_TIMEOUT", 5: "ERR_CUDA",
          6: "ERR_IO", 7: "ERR_STATE", 8: "ERR_OVERFLOW", 9: "ERR_INTERNAL"}
PHASES = ("filter", "index", "tables", "join", "total", "h2d", "d2h", "host")

# C-ABI symbols declared in include/gem.h (checked by the CPU test suite).
EXPORTS = (
    "gem_strerror", "gem_hgraph_create", "gem_hgraph_read_text", "gem_hgraph_write_text",
    "gem_hgraph_rmat", "gem_hgraph_set_labels", "gem_hgraph_info", "gem_hgraph_view",
    "gem_hgraph_destroy", "gem_query_read_text", "gem_query_write_text", "gem_gen_queries",
    "gem_ctx_create", "gem_ctx_destroy", "gem_last_error", "gem_ctx_load_graph", "gem_query_run",
    "gem_batch_run", "gem_embedding_hash", "gem_filter", "gem_edge_table", "gem_index_probe",
    "gem_submit", "gem_poll", "gem_autotune", "gem_filter_static", "gem_set_schedule", "gem_get_schedule",
    "gem_relaxed_sets", "gem_relaxed_run", "gem_ctx_ooc_stats", "gem_plan_query", "gem_hgraph_partitions",
    "gem_estimate_bytes",
)


class GemError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


class _Query(C.Structure):
    _fields_ = [("nv", C.c_uint32), ("ne", C.c_uint32), ("labels", C.POINTER(C.c_uint32)),
                ("edges", C.POINTER(C.c_uint32))]


class _Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("device_budget_bytes", C.c_uint64), ("pinned_budget_bytes", C.c_uint64),
                ("ooc", C.c_int), ("time_cap_ms", C.c_uint32), ("index_kind", C.c_uint32),
                ("admit_gb", C.c_uint32), ("ooc_part_kib", C.c_uint32), ("ooc_stream", C.c_uint32),
                ("batch_lanes", C.c_uint32), ("reserved", C.c_uint32 * 2)]


class _OocStats(C.Structure):
    _fields_ = [("partitions", C.c_uint32), ("reserved0", C.c_uint32), ("max_part_bytes", C.c_uint64),
                ("waves_streamed", C.c_uint64), ("waves_in_place", C.c_uint64), ("parts_streamed", C.c_uint64),
                ("bytes_streamed", C.c_uint64), ("waves_spilled", C.c_uint64), ("bytes_spilled", C.c_uint64),
                ("resident_bytes", C.c_uint64)]


class _Schedule(C.Structure):
    _fields_ = [("blocks_per_sm", C.c_uint32), ("donate_max_level", C.c_uint32), ("donate_min_lane", C.c_uint32),
                ("donate_min_desc", C.c_uint32), ("root_batch_max", C.c_uint32), ("lane_scan_max", C.c_uint32),
                ("split_blocks", C.c_uint32), ("reserved", C.c_uint32)]


SCHEDULE_FIELDS = ("blocks_per_sm", "donate_max_level", "donate_min_lane", "donate_min_desc", "root_batch_max",
                   "lane_scan_max", "split_blocks")


class _Result(C.Structure):
    _fields_ = [("count", C.c_uint64), ("emb_hash", C.c_uint64), ("n_written", C.c_uint64),
                ("status", C.c_uint32), ("n_tables", C.c_uint32), ("cand_total", C.c_uint64),
                ("table_total", C.c_uint64), ("nodes", C.c_uint64), ("bytes_alg", C.c_uint64 * 4),
                ("ms", C.c_float * 8), ("wave", C.c_uint32), ("launches", C.c_uint32),
                ("table_pass_ms", C.c_float * 2), ("t_begin_ms", C.c_float), ("t_end_ms", C.c_float),
                ("arena_bytes", C.c_uint64)]


_lib = None


def lib():
    """Load libgem.so (built in-tree by gem_b200.build / __graft_entry__.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgem.so not built at {LIB_PATH}; run `python -m gem_b200.build`")
        L = C.CDLL(LIB_PATH)
        u32p, u64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
        vp = C.c_void_p
        L.gem_strerror.restype = C.c_char_p
        L.gem_last_error.restype = C.c_char_p
        L.gem_last_error.argtypes = [vp]
        L.gem_hgraph_create.argtypes = [C.c_uint32, u64p, u32p, u32p, C.POINTER(vp)]
        L.gem_hgraph_read_text.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.gem_hgraph_write_text.argtypes = [vp, C.c_char_p]
        L.gem_hgraph_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                      C.POINTER(vp)]
        L.gem_hgraph_set_labels.argtypes = [vp, C.c_uint32, C.c_double, C.c_uint64]
        L.gem_hgraph_info.argtypes = [vp, u32p, u64p, u32p, u32p]
        L.gem_hgraph_view.argtypes = [vp, C.POINTER(u64p), C.POINTER(u32p), C.POINTER(u32p)]
        L.gem_hgraph_destroy.argtypes = [vp]
        L.gem_hgraph_destroy.restype = None
        L.gem_query_read_text.argtypes = [C.c_char_p, u32p, u32p, u32p, u32p]
        L.gem_query_write_text.argtypes = [C.POINTER(_Query), C.c_char_p]
        L.gem_gen_queries.argtypes = [vp, C.c_uint32, C.c_int, C.c_uint32, C.c_uint64, C.c_uint32, u32p, u32p, u32p]
        L.gem_ctx_create.argtypes = [C.POINTER(_Opts), C.POINTER(vp)]
        L.gem_ctx_destroy.argtypes = [vp]
        L.gem_ctx_destroy.restype = None
        L.gem_ctx_load_graph.argtypes = [vp, vp]
        L.gem_query_run.argtypes = [vp, C.POINTER(_Query), C.c_uint32, C.c_int, u32p, C.c_uint64,
                                    C.POINTER(_Result)]
        L.gem_batch_run.argtypes = [vp, C.POINTER(_Query), C.c_uint32, C.c_int, C.POINTER(_Result)]
        L.gem_embedding_hash.argtypes = [u32p, C.c_uint32]
        L.gem_embedding_hash.restype = C.c_uint64
        L.gem_filter.argtypes = [vp, C.POINTER(_Query), C.c_uint32, u32p, u32p, C.c_uint64]
        L.gem_edge_table.argtypes = [vp, C.POINTER(_Query), C.c_uint32, C.c_uint32, u64p, C.c_uint64, u32p,
                                     C.c_uint64, u64p, u64p]
        L.gem_index_probe.argtypes = [vp, C.POINTER(_Query), C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p]
        L.gem_submit.argtypes = [vp, C.POINTER(_Query), C.c_int, u64p]
        L.gem_estimate_bytes.argtypes = [vp, C.POINTER(_Query), u64p]
        L.gem_poll.argtypes = [vp, C.c_uint64, C.POINTER(_Result), C.POINTER(C.c_int)]
        L.gem_autotune.argtypes = [vp, C.POINTER(_Query), C.c_uint32, C.c_int, C.c_uint32, u32p]
        L.gem_relaxed_sets.argtypes = [C.POINTER(_Query), C.c_uint32, C.c_uint32, u64p, u32p]
        L.gem_relaxed_run.argtypes = [vp, C.POINTER(_Query), C.c_uint32, C.c_int, C.c_uint32, u64p,
                                      C.POINTER(_Result), u32p]
        L.gem_set_schedule.argtypes = [vp, C.c_uint32, C.POINTER(_Schedule)]
        L.gem_get_schedule.argtypes = [vp, C.c_uint32, C.POINTER(_Schedule)]
        L.gem_ctx_ooc_stats.argtypes = [vp, C.POINTER(_OocStats)]
        L.gem_plan_query.argtypes = [C.POINTER(_Query), u32p, C.c_int, u32p, u32p]
        L.gem_hgraph_partitions.argtypes = [vp, C.c_uint32, u32p, C.c_uint32, u32p]
        L.gem_filter_static.argtypes = [vp, vp, vp, C.c_uint32, C.POINTER(_Query), C.c_uint32, u32p, vp,
                                        C.c_uint64, vp]
        _lib = L
    return _lib


def _p32(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _check(st, ctx=None, what=""):
    if st != 0:
        msg = what
        if ctx is not None:
            m = lib().gem_last_error(ctx)
            if m:
                msg += ": " + m.decode()
        raise GemError(st, msg)


class Query:
    """A query graph: labels (nv,) and undirected edges (ne, 2), vertices 0..nv-1."""

    def __init__(self, labels, edges):
        self.labels = np.ascontiguousarray(np.asarray(labels, dtype=np.uint32).reshape(-1))
        e = np.asarray(edges, dtype=np.uint32).reshape(-1, 2) if len(edges) else np.zeros((0, 2), np.uint32)
        self.edges = np.ascontiguousarray(e)

    @property
    def nv(self):
        return int(self.labels.shape[0])

    @property
    def ne(self):
        return int(self.edges.shape[0])

    def _c(self):
        # built once: the pointers refer to this object's arrays, which it keeps
        cq = self.__dict__.get("_cq")
        if cq is None:
            self._flat_edges = self.edges.reshape(-1)
            cq = _Query(self.nv, self.ne, _p32(self.labels), _p32(self._flat_edges))
            self._cq = cq
        return cq

    @staticmethod
    def read_text(path):
        nv, ne = C.c_uint32(), C.c_uint32()
        lab = np.zeros(MAX_QV, np.uint32)
        edg = np.zeros(2 * MAX_QE, np.uint32)
        _check(lib().gem_query_read_text(path.encode(), C.byref(nv), C.byref(ne), _p32(lab), _p32(edg)),
               what=f"read {path}")
        return Query(lab[:nv.value].copy(), edg[:2 * ne.value].reshape(-1, 2).copy())

    def write_text(self, path):
        q = self._c()
        _check(lib().gem_query_write_text(C.byref(q), path.encode()), what=f"write {path}")

    def __repr__(self):
        return f"Query(nv={self.nv}, ne={self.ne})"


class HostGraph:
    """Host CSR data graph with sorted adjacency (owned by libgem)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.gem_hgraph_destroy(self._h)
            self._h = C.c_void_p(0)

    @staticmethod
    def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=None):
        h = C.c_void_p()
        seed = (0x47454D00 + scale) if seed is None else seed
        _check(lib().gem_hgraph_rmat(scale, edge_factor, a, b, c, seed, C.byref(h)), what="rmat")
        return HostGraph(h)

    @staticmethod
    def from_csr(offsets, nbrs, labels):
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nb = np.ascontiguousarray(nbrs, dtype=np.uint32)
        lb = np.ascontiguousarray(labels, dtype=np.uint32)
        if nb.size == 0:
            nb = np.zeros(1, np.uint32)
        h = C.c_void_p()
        _check(lib().gem_hgraph_create(len(lb), _p64(off), _p32(nb), _p32(lb), C.byref(h)), what="hgraph_create")
        return HostGraph(h)

    @staticmethod
    def from_edges(nv, edges, labels):
        """Undirected edge list -> CSR with sorted adjacency."""
        e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
        e = e[e[:, 0] != e[:, 1]]
        lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
        key = np.unique(lo * (nv + 1) + hi)
        lo, hi = key // (nv + 1), key % (nv + 1)
        src = np.concatenate([lo, hi])
        dst = np.concatenate([hi, lo])
        order = np.lexsort((dst, src))
        src, dst = src[order], dst[order]
        off = np.zeros(nv + 1, np.uint64)
        np.add.at(off, src + 1, 1)
        off = np.cumsum(off).astype(np.uint64)
        return HostGraph.from_csr(off, dst.astype(np.uint32), labels)

    @staticmethod
    def read_text(path):
        h = C.c_void_p()
        _check(lib().gem_hgraph_read_text(path.encode(), C.byref(h)), what=f"read {path}")
        return HostGraph(h)

    def write_text(self, path):
        _check(lib().gem_hgraph_write_text(self._h, path.encode()), what=f"write {path}")

    def set_labels(self, nlabels, zipf_s=0.0, seed=None):
        if seed is None:
            seed = 0x47454D4C
        _check(lib().gem_hgraph_set_labels(self._h, nlabels, zipf_s, seed), what="set_labels")
        return self

    def partitions(self, part_kib=0):
        """Vertex bounds of the out-of-core adjacency partitions (gem_hgraph_partitions; part_kib 0 = 16 MiB)."""
        n = C.c_uint32()
        st = lib().gem_hgraph_partitions(self._h, part_kib, None, 0, C.byref(n))
        if st not in (0, 3):
            _check(st, what="partitions")
        out = np.zeros(n.value + 1, np.uint32)
        _check(lib().gem_hgraph_partitions(self._h, part_kib, _p32(out), n.value + 1, C.byref(n)), what="partitions")
        return out

    def info(self):
        nv, na, ml, md = C.c_uint32(), C.c_uint64(), C.c_uint32(), C.c_uint32()
        _check(lib().gem_hgraph_info(self._h, C.byref(nv), C.byref(na), C.byref(ml), C.byref(md)))
        return {"nv": nv.value, "n_arcs": na.value, "n_labels": ml.value, "max_degree": md.value}

    @property
    def nv(self):
        return self.info()["nv"]

    def arrays(self):
        """(offsets u64[nv+1], nbrs u32[arcs], labels u32[nv]) as read-only numpy views."""
        inf = self.info()
        po, pn, pl = C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
        _check(lib().gem_hgraph_view(self._h, C.byref(po), C.byref(pn), C.byref(pl)))
        off = np.ctypeslib.as_array(po, shape=(inf["nv"] + 1,))
        nbr = np.ctypeslib.as_array(pn, shape=(max(inf["n_arcs"], 1),))[:inf["n_arcs"]]
        lab = np.ctypeslib.as_array(pl, shape=(max(inf["nv"], 1),))[:inf["nv"]]
        for a in (off, nbr, lab):
            a.flags.writeable = False
        return off, nbr, lab


def gen_queries(graph, k, density=ANY, count=1, seed=0x51000, max_e=MAX_QE):
    """Random-walk queries (see gem_gen_queries in include/gem.h)."""
    ne = np.zeros(count, np.uint32)
    lab = np.zeros(count * k, np.uint32)
    edg = np.zeros(count * 2 * max_e, np.uint32)
    _check(lib().gem_gen_queries(graph._h, k, density, count, seed, max_e, _p32(ne), _p32(lab), _p32(edg)),
           what="gen_queries")
    out = []
    for i in range(count):
        e = edg[i * 2 * max_e: i * 2 * max_e + 2 * int(ne[i])].reshape(-1, 2).copy()
        out.append(Query(lab[i * k:(i + 1) * k].copy(), e))
    return out


def relaxed_sets(q, threshold, cap=4096):
    """Edge masks (bit j = edge j of q kept) of q's relaxed queries at `threshold` (gem_relaxed_sets)."""
    ets = np.zeros(max(cap, 1), np.uint64)
    n = C.c_uint32()
    qc = q._c()
    _check(lib().gem_relaxed_sets(C.byref(qc), threshold, cap, _p64(ets), C.byref(n)), what="relaxed_sets")
    return [int(x) for x in ets[:n.value]]


def plan(q, cand_counts, closed_form=True):
    """Matching order of q given |C(u)| per query vertex (gem_plan_query): (n_enum, order), order[k] the
    query vertex of level k; with closed_form, levels n_enum.. are counted in closed form."""
    cnt = np.ascontiguousarray(cand_counts, dtype=np.uint32)
    if len(cnt) < q.nv:
        raise ValueError("one candidate count per query vertex")
    order = np.zeros(max(q.nv, 1), np.uint32)
    ne = C.c_uint32()
    qc = q._c()
    _check(lib().gem_plan_query(C.byref(qc), _p32(cnt), 1 if closed_form else 0, C.byref(ne), _p32(order)),
           what="plan")
    return ne.value, order[:q.nv].tolist()


def relaxed_query(q, et):
    """The relaxed query of q that keeps the edges in mask et."""
    keep = [e for j, e in enumerate(q.edges.tolist()) if (et >> j) & 1]
    return Query(q.labels, keep)


def embedding_hash(f):
    f = np.ascontiguousarray(f, dtype=np.uint32)
    return int(lib().gem_embedding_hash(_p32(f), len(f)))


class Result(dict):
    """Per-query result: count, emb_hash, status, timings (ms) and byte counters."""

    @staticmethod
    def _from(r):
        d = Result(count=int(r.count), emb_hash=int(r.emb_hash), n_written=int(r.n_written),
                   status=STATUS.get(r.status, r.status), status_code=int(r.status), n_tables=int(r.n_tables),
                   cand_total=int(r.cand_total), table_total=int(r.table_total), nodes=int(r.nodes),
                   bytes_alg=[int(x) for x in r.bytes_alg], ms={p: float(r.ms[i]) for i, p in enumerate(PHASES)},
                   wave=int(r.wave), launches=int(r.launches),
                   table_pass_ms=[float(r.table_pass_ms[0]), float(r.table_pass_ms[1])],
                   t_begin_ms=float(r.t_begin_ms), t_end_ms=float(r.t_end_ms), arena_bytes=int(r.arena_bytes))
        return d


class Context:
    """One GPU with a resident data graph (gem_ctx)."""

    def __init__(self, device=0, budget_bytes=0, time_cap_ms=0, index_kind=IDX_AUTO, ooc=False, pinned_bytes=0,
                 admit_gb=0, ooc_part_kib=0, ooc_stream=0, batch_lanes=0):
        """ooc_part_kib / ooc_stream: out-of-core adjacency partition size (KiB, 0 = 16 MiB) and whether
        table builds stream partitions (0 = when the sources fill them enough, 1 = always, 2 = never)."""
        o = _Opts()
        o.admit_gb = admit_gb
        o.ooc_part_kib = ooc_part_kib
        o.ooc_stream = ooc_stream
        o.batch_lanes = batch_lanes
        o.device = device
        o.device_budget_bytes = budget_bytes
        o.pinned_budget_bytes = pinned_bytes
        o.ooc = 1 if ooc else 0
        o.time_cap_ms = time_cap_ms
        o.index_kind = index_kind
        h = C.c_void_p()
        _check(lib().gem_ctx_create(C.byref(o), C.byref(h)), what="ctx_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gem_ctx_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def load_graph(self, g):
        _check(lib().gem_ctx_load_graph(self._h, g._h), self._h, "load_graph")

    def run(self, q, mode=MODE_COUNT, threshold=0, emb_cap=0, raise_on_error=True):
        qc = q._c()
        r = _Result()
        buf = np.zeros(max(emb_cap, 1) * q.nv, np.uint32) if mode == MODE_ENUMERATE else None
        st = lib().gem_query_run(self._h, C.byref(qc), threshold, mode, _p32(buf) if buf is not None else None,
                                 emb_cap, C.byref(r))
        res = Result._from(r)
        if st != 0 and res["status_code"] == 0:
            res["status"], res["status_code"] = STATUS.get(st, st), st
        if st != 0:
            m = lib().gem_last_error(self._h)
            res["error"] = m.decode() if m else ""
        if mode == MODE_ENUMERATE:
            res["embeddings"] = buf[: res["n_written"] * q.nv].reshape(-1, q.nv)
        if st != 0 and raise_on_error and st != 8:
            _check(st, self._h, "query_run")
        return res

    def batch(self, qs, mode=MODE_COUNT):
        arr = (_Query * len(qs))()
        keep = []
        for i, q in enumerate(qs):
            arr[i] = q._c()
            keep.append(q)
        rs = (_Result * len(qs))()
        st = lib().gem_batch_run(self._h, arr, len(qs), mode, rs)
        out = [Result._from(r) for r in rs]
        if st != 0:
            m = lib().gem_last_error(self._h)
            for r in out:
                r["error"] = m.decode() if m else ""
        return st, out

    def relaxed(self, q, threshold, mode=MODE_COUNT, cap=4096):
        """Relaxed matching (gem_relaxed_run): [(edge mask, Result)] for q's relaxed queries."""
        ets = np.zeros(max(cap, 1), np.uint64)
        rs = (_Result * max(cap, 1))()
        n = C.c_uint32()
        qc = q._c()
        st = lib().gem_relaxed_run(self._h, C.byref(qc), threshold, mode, cap, _p64(ets), rs, C.byref(n))
        _check(st, self._h, "relaxed")
        return [(int(ets[i]), Result._from(rs[i])) for i in range(n.value)]

    def batch_counts(self, qs, mode=MODE_COUNT):
        """gem_batch_run without per-query dicts: (status, counts u64[n], statuses i32[n])."""
        n = len(qs)
        arr = (_Query * n)()
        for i, q in enumerate(qs):
            arr[i] = q._c()
        rs = (_Result * n)()
        st = lib().gem_batch_run(self._h, arr, n, mode, rs)
        raw = np.frombuffer(rs, dtype=np.uint8).reshape(n, C.sizeof(_Result))
        counts = raw[:, _Result.count.offset:_Result.count.offset + 8].copy().view(np.uint64).reshape(n)
        status = raw[:, _Result.status.offset:_Result.status.offset + 4].copy().view(np.int32).reshape(n)
        return st, counts, status

    def autotune(self, qs, mode=MODE_COUNT, trial_cap_ms=2000):
        """Tune the join schedule per query-size bucket; returns {bucket: (blocks/SM, donate level, us)}."""
        arr = (_Query * max(len(qs), 1))()
        for i, q in enumerate(qs):
            arr[i] = q._c()
        rep = np.zeros(18, np.uint32)
        _check(lib().gem_autotune(self._h, arr, len(qs), mode, trial_cap_ms, _p32(rep)), self._h, "autotune")
        names = ("<=4", "<=8", "<=12", "<=16", "<=24", "<=32")
        out = {}
        for b in range(6):
            if rep[3 * b]:
                sched = int(rep[3 * b + 1])
                out[names[b]] = {"blocks_per_sm": int(rep[3 * b]), "donate_max_level": sched & 0xFF,
                                 "donate_min_lane": (sched >> 8) & 0xFFF, "root_batch_max": sched >> 20,
                                 "join_us": int(rep[3 * b + 2])}
        return out

    def set_schedule(self, query_vertices, **fields):
        """Pin the join schedule of a query-size bucket (fields of gem_schedule; 0 = default)."""
        sc = _Schedule()
        for k, v in fields.items():
            if k not in SCHEDULE_FIELDS:
                raise ValueError(f"unknown schedule field {k}")
            setattr(sc, k, int(v))
        _check(lib().gem_set_schedule(self._h, query_vertices, C.byref(sc)), self._h, "set_schedule")

    def get_schedule(self, query_vertices):
        sc = _Schedule()
        _check(lib().gem_get_schedule(self._h, query_vertices, C.byref(sc)), self._h, "get_schedule")
        return {k: int(getattr(sc, k)) for k in SCHEDULE_FIELDS}

    def ooc_stats(self):
        """Out-of-core partition streaming counters since the graph was loaded (gem_ctx_ooc_stats)."""
        st = _OocStats()
        _check(lib().gem_ctx_ooc_stats(self._h, C.byref(st)), self._h, "ooc_stats")
        return {k: int(getattr(st, k)) for k, _ in _OocStats._fields_ if k != "reserved0"}

    def estimate_bytes(self, q):
        """Device scratch bytes serving admission reserves for q (gem_estimate_bytes)."""
        b = C.c_uint64()
        qc = q._c()
        _check(lib().gem_estimate_bytes(self._h, C.byref(qc), C.byref(b)), self._h, "estimate_bytes")
        return b.value

    def submit(self, q, mode=MODE_COUNT):
        """Serving: returns a ticket, or None when admission is busy (retry later)."""
        qc = q._c()
        t = C.c_uint64()
        st = lib().gem_submit(self._h, C.byref(qc), mode, C.byref(t))
        if st == 2:
            return None
        _check(st, self._h, "submit")
        return t.value

    def poll(self, ticket):
        """Serving: the Result of `ticket` once done, else None."""
        r = _Result()
        done = C.c_int()
        _check(lib().gem_poll(self._h, ticket, C.byref(r), C.byref(done)), self._h, "poll")
        return Result._from(r) if done.value else None

    def filter(self, q, threshold=0):
        counts = np.zeros(q.nv, np.uint32)
        cap = 1 << 26
        cand = np.zeros(cap, np.uint32)
        qc = q._c()
        _check(lib().gem_filter(self._h, C.byref(qc), threshold, _p32(counts), _p32(cand), cap), self._h, "filter")
        lists, at = [], 0
        for u in range(q.nv):
            lists.append(cand[at:at + int(counts[u])].copy())
            at += int(counts[u])
        return lists

    def edge_table(self, q, u, w, values_cap=1 << 26):
        nk, nvals = C.c_uint64(), C.c_uint64()
        off = np.zeros(1 << 24, np.uint64)
        vals = np.zeros(values_cap, np.uint32)
        qc = q._c()
        _check(lib().gem_edge_table(self._h, C.byref(qc), u, w, _p64(off), off.size, _p32(vals), values_cap,
                                    C.byref(nk), C.byref(nvals)), self._h, "edge_table")
        return off[:nk.value + 1].copy(), vals[:nvals.value].copy()

    def index_probe(self, q, u, keys, kind=IDX_RANK):
        keys = np.ascontiguousarray(keys, dtype=np.uint32)
        out = np.zeros(max(len(keys), 1), np.uint32)
        qc = q._c()
        _check(lib().gem_index_probe(self._h, C.byref(qc), u, kind, _p32(keys), len(keys), _p32(out)), self._h,
               "index_probe")
        return out[:len(keys)]
