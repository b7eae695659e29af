"""GPU path (libgem, sm_100a) against the CPU oracle and the golden fixtures.
Bit-exact: integer counts, candidate lists, tables and hashes must be equal."""
import json
import os

import numpy as np
import pytest

import gem_b200 as gem
import oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cases.json")


def cases():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def small():
    # config-1 shape at reduced size: R-MAT scale 12, edge factor 8, 4 uniform labels
    g = gem.HostGraph.rmat(12, 8, seed=0x47454D00 + 12).set_labels(4, 0.0, seed=0x47454D0C ^ 0x4C)
    return g


@pytest.fixture(scope="module")
def gctx(small):
    c = gem.Context(time_cap_ms=30000)
    c.load_graph(small)
    yield c
    c.close()


@pytest.mark.parametrize("case", cases(), ids=lambda c: c["name"])
def test_golden_counts_and_hash(case):
    g = gem.HostGraph.from_edges(case["nv"], case["edges"], case["labels"])
    q = gem.Query(case["qlabels"], case["qedges"])
    with gem.Context(time_cap_ms=20000) as c:
        c.load_graph(g)
        r = c.run(q, mode=gem.MODE_HASH)
    assert r["status"] == "OK"
    assert r["count"] == case["count"]
    assert r["emb_hash"] == int(case["hash"])


def test_filter_matches_oracle(small, gctx):
    for k, dens in ((4, gem.ANY), (8, gem.SPARSE), (8, gem.DENSE), (16, gem.ANY)):
        for q in gem.gen_queries(small, k, dens, 3, seed=100 + k):
            for T in (0, 1, 2):
                got = gctx.filter(q, threshold=T)
                exp = oracle.filter(small, q, threshold=T)
                for u in range(q.nv):
                    assert np.array_equal(got[u], exp[u]), (k, T, u)


def test_edge_tables_match_oracle(small, gctx):
    for q in gem.gen_queries(small, 6, gem.ANY, 3, seed=5):
        cand = oracle.filter(small, q)
        for a, b in q.edges.tolist():
            for u, w in ((a, b), (b, a)):
                off, vals = gctx.edge_table(q, u, w)
                eo, ev = oracle.edge_table(small, cand[u], cand[w])
                assert np.array_equal(off, eo), (u, w)
                assert np.array_equal(vals, ev), (u, w)


@pytest.mark.parametrize("kind", [gem.IDX_RANK, gem.IDX_CUCKOO])
def test_index_probe_positions(small, gctx, kind):
    for q in gem.gen_queries(small, 5, gem.ANY, 2, seed=9):
        cand = oracle.filter(small, q)
        for u in range(q.nv):
            keys = cand[u]
            pos = gctx.index_probe(q, u, keys, kind=kind)
            assert np.array_equal(pos, np.arange(len(keys), dtype=np.uint32))
            # absent keys report 0xFFFFFFFF
            absent = np.setdiff1d(np.arange(0, small.nv, 7, dtype=np.uint32), keys)[:200]
            if len(absent):
                assert np.all(gctx.index_probe(q, u, absent, kind=kind) == 0xFFFFFFFF)


def test_cuckoo_large_table():
    # one label: every vertex is a candidate -> table far above the shared-memory path
    g = gem.HostGraph.rmat(15, 4, seed=3).set_labels(1)
    q = gem.Query([0, 0], [(0, 1)])
    with gem.Context(time_cap_ms=20000) as c:
        c.load_graph(g)
        cand = oracle.filter(g, q)[0]
        pos = c.index_probe(q, 0, cand, kind=gem.IDX_CUCKOO)
        assert np.array_equal(pos, np.arange(len(cand), dtype=np.uint32))


@pytest.mark.parametrize("k,dens,n", [(3, gem.ANY, 6), (4, gem.ANY, 8), (5, gem.SPARSE, 6), (6, gem.DENSE, 6),
                                      (8, gem.SPARSE, 4), (8, gem.DENSE, 4)])
def test_counts_match_oracle(small, gctx, k, dens, n):
    for q in gem.gen_queries(small, k, dens, n, seed=1000 + k * 10 + dens):
        exp, eh, ok = oracle.count(small, q, threads=0, work_cap=400_000_000)
        if not ok:
            continue
        r = gctx.run(q, mode=gem.MODE_HASH)
        assert r["status"] == "OK"
        assert r["count"] == exp, (q.labels.tolist(), q.edges.tolist())
        assert r["emb_hash"] == eh
        rc = gctx.run(q, mode=gem.MODE_COUNT)
        assert rc["count"] == exp


@pytest.mark.parametrize("kind", [gem.IDX_RANK, gem.IDX_CUCKOO])
def test_index_kinds_same_counts(small, kind):
    with gem.Context(index_kind=kind, time_cap_ms=30000) as c:
        c.load_graph(small)
        for q in gem.gen_queries(small, 5, gem.ANY, 4, seed=31):
            exp, eh, ok = oracle.count(small, q, work_cap=400_000_000)
            if ok:
                r = c.run(q, mode=gem.MODE_HASH)
                assert (r["count"], r["emb_hash"]) == (exp, eh)


def test_enumerate_embeddings(small, gctx):
    for q in gem.gen_queries(small, 4, gem.ANY, 3, seed=77):
        exp, eh, ok = oracle.count(small, q)
        if not ok or exp > 2_000_000:
            continue
        r = gctx.run(q, mode=gem.MODE_ENUMERATE, emb_cap=exp + 10)
        assert r["count"] == exp and r["n_written"] == exp and r["emb_hash"] == eh
        emb = r["embeddings"]
        # every row is a valid embedding, rows are distinct, hashes add up
        off, nbr, lab = small.arrays()
        assert np.all(lab[emb] == q.labels[None, :])
        for a, b in q.edges.tolist():
            x, y = emb[:, a].astype(np.int64), emb[:, b].astype(np.int64)
            s = np.searchsorted(nbr[:0], [])  # noqa: keep numpy happy on empty
            for i in range(0, len(emb), max(1, len(emb) // 200)):
                lst = nbr[off[x[i]]:off[x[i] + 1]]
                assert y[i] in lst
        assert len(np.unique(emb, axis=0)) == len(emb)
        h = 0
        for row in emb[: min(len(emb), 3000)]:
            h = (h + gem.embedding_hash(row)) % (1 << 64)
        if len(emb) <= 3000:
            assert h == eh


def test_enumerate_overflow_keeps_exact_count(small, gctx):
    q = gem.gen_queries(small, 4, gem.ANY, 1, seed=5)[0]
    exp, _, ok = oracle.count(small, q)
    assert ok and exp > 10
    r = gctx.run(q, mode=gem.MODE_ENUMERATE, emb_cap=10)
    assert r["status"] == "ERR_OVERFLOW" and r["count"] == exp and r["n_written"] == 10


def test_batch_equals_plain(small, gctx):
    qs = []
    for k in (2, 3, 4, 5, 6, 8):
        for q in gem.gen_queries(small, k, gem.ANY, 6, seed=500 + k):
            if oracle.count(small, q, want_hash=False, work_cap=200_000_000)[2]:
                qs.append(q)
    assert len(qs) >= 12
    plain = [gctx.run(q, mode=gem.MODE_HASH) for q in qs]
    st, batch = gctx.batch(qs, mode=gem.MODE_HASH)
    assert st == 0
    for p, b in zip(plain, batch):
        assert (p["count"], p["emb_hash"]) == (b["count"], b["emb_hash"])


def test_edge_cases(small, gctx):
    off, nbr, lab = small.arrays()
    # single vertex: count = vertices with that label
    q1 = gem.Query([lab[0]], [])
    assert gctx.run(q1)["count"] == int(np.sum(lab == lab[0]))
    # label absent from the data graph: 0
    assert gctx.run(gem.Query([0, 99], [(0, 1)]))["count"] == 0
    # single edge (the reference prints no result for |E_q| <= 1)
    q2 = gem.Query([0, 1], [(0, 1)])
    exp, _, _ = oracle.count(small, q2)
    assert gctx.run(q2)["count"] == exp
    # same-label star (injectivity among leaves)
    q3 = gem.Query([0, 0, 0, 0], [(0, 1), (0, 2), (0, 3)])
    exp, eh, ok = oracle.count(small, q3, work_cap=500_000_000)
    if ok:
        r = gctx.run(q3, mode=gem.MODE_HASH)
        assert (r["count"], r["emb_hash"]) == (exp, eh)
    # invalid queries are rejected on the host
    with pytest.raises(gem.GemError):
        gctx.run(gem.Query([0, 1, 2], [(0, 1)]))  # disconnected
    with pytest.raises(gem.GemError):
        gctx.run(gem.Query([0, 1], [(0, 0)]))  # self loop
    with pytest.raises(gem.GemError):
        gctx.run(gem.Query([0, 1], [(0, 1)]), threshold=1)


def test_max_size_queries(tiny):
    with gem.Context(time_cap_ms=20000) as c:
        c.load_graph(tiny)
        done = 0
        for q in gem.gen_queries(tiny, 32, gem.DENSE, 4, seed=3210):
            assert q.nv == 32
            exp, eh, ok = oracle.count(tiny, q, work_cap=300_000_000)
            if not ok:
                continue
            r = c.run(q, mode=gem.MODE_HASH, raise_on_error=False)
            assert r["status"] in ("OK", "ERR_TIMEOUT")
            if r["status"] == "OK":
                assert (r["count"], r["emb_hash"]) == (exp, eh)
                assert c.run(q)["count"] == exp
                done += 1


def test_time_cap_reports_timeout():
    g = gem.HostGraph.rmat(16, 16, seed=1).set_labels(1)
    q = gem.Query([0] * 6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5)])
    with gem.Context(time_cap_ms=50) as c:
        c.load_graph(g)
        r = c.run(q, raise_on_error=False)
        assert r["status"] == "ERR_TIMEOUT"
        # the context stays usable after a timeout
        r2 = c.run(gem.Query([0], []))
        assert r2["status"] == "OK" and r2["count"] == g.nv


SUFFIX_SHAPES = {
    # name: (labels, edges)
    "star4_same": ([0, 1, 1, 1, 1], [(0, 1), (0, 2), (0, 3), (0, 4)]),
    "star3_mixed": ([0, 1, 1, 2], [(0, 1), (0, 2), (0, 3)]),
    "star3_all_same": ([1, 1, 1, 1], [(0, 1), (0, 2), (0, 3)]),
    "double_star": ([0, 0, 1, 1, 1, 1], [(0, 1), (0, 2), (0, 3), (1, 4), (1, 5)]),
    "path5_same": ([1, 1, 1, 1, 1], [(0, 1), (1, 2), (2, 3), (3, 4)]),
    "cycle4_leaves": ([0, 1, 0, 1, 2, 2], [(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (2, 5)]),
    "triangle_tail": ([0, 0, 1, 1], [(0, 1), (1, 2), (2, 0), (2, 3)]),
    "k4_leaves": ([0, 1, 2, 0, 1, 1], [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (3, 4), (0, 5)]),
    "two_parents_same_leaf_label": ([0, 1, 2, 2, 2], [(0, 1), (0, 2), (1, 3), (1, 4), (0, 4)]),
}


@pytest.fixture(scope="module")
def tiny():
    return gem.HostGraph.rmat(10, 8, seed=77).set_labels(3, 0.0, seed=78)


@pytest.mark.parametrize("shape", sorted(SUFFIX_SHAPES))
def test_closed_form_suffix_shapes(tiny, shape):
    labels, edges = SUFFIX_SHAPES[shape]
    q = gem.Query(labels, edges)
    exp, eh, ok = oracle.count(tiny, q, work_cap=2_000_000_000)
    assert ok
    with gem.Context(time_cap_ms=30000) as c:
        c.load_graph(tiny)
        rc = c.run(q, mode=gem.MODE_COUNT)
        rh = c.run(q, mode=gem.MODE_HASH)
    assert rc["count"] == exp, (shape, rc["count"], exp)
    assert (rh["count"], rh["emb_hash"]) == (exp, eh)


def test_suffix_random_queries_tiny(tiny):
    for k in (3, 4, 5, 6, 7):
        for d in (gem.SPARSE, gem.ANY):
            for q in gem.gen_queries(tiny, k, d, 5, seed=900 + 10 * k + d):
                exp, _, ok = oracle.count(tiny, q, want_hash=False, work_cap=500_000_000)
                if not ok:
                    continue
                with gem.Context(time_cap_ms=30000) as c:
                    c.load_graph(tiny)
                    assert c.run(q)["count"] == exp, (q.labels.tolist(), q.edges.tolist())


def test_serving_matches_plain(small):
    qs = []
    for k in (3, 4, 5):
        for q in gem.gen_queries(small, k, gem.ANY, 8, seed=4000 + k):
            if oracle.count(small, q, want_hash=False, work_cap=100_000_000)[2]:
                qs.append(q)
    with gem.Context(time_cap_ms=30000) as plain_ctx:
        plain_ctx.load_graph(small)
        alone = [plain_ctx.run(q, mode=gem.MODE_HASH) for q in qs]
    import random
    import time
    rng = random.Random(5)
    with gem.Context(time_cap_ms=30000) as srv:
        srv.load_graph(small)
        tickets, pending, results = {}, list(range(len(qs))), {}
        # staggered arrivals: submit a few, poll, submit more while waves run
        while pending or tickets:
            for _ in range(rng.randint(1, 4)):
                if pending:
                    i = pending.pop(0)
                    t = srv.submit(qs[i], mode=gem.MODE_HASH)
                    if t is None:
                        pending.insert(0, i)
                        break
                    tickets[t] = i
            for t in list(tickets):
                r = srv.poll(t)
                if r is not None:
                    results[tickets.pop(t)] = r
            time.sleep(0.001)
        with pytest.raises(gem.GemError):
            srv.run(qs[0])  # the serving context accepts only submit/poll
    waves = {r["wave"] for r in results.values()}
    for i, a in enumerate(alone):
        assert (results[i]["count"], results[i]["emb_hash"]) == (a["count"], a["emb_hash"])
    assert len(waves) >= 1


def test_out_of_core_same_counts(small):
    qs = [q for q in gem.gen_queries(small, 5, gem.ANY, 6, seed=6100)
          if oracle.count(small, q, want_hash=False, work_cap=100_000_000)[2]]
    with gem.Context(time_cap_ms=30000) as a, gem.Context(time_cap_ms=30000, ooc=True, budget_bytes=2 << 30) as b:
        a.load_graph(small)
        b.load_graph(small)
        for q in qs:
            ra, rb = a.run(q, mode=gem.MODE_HASH), b.run(q, mode=gem.MODE_HASH)
            assert (ra["count"], ra["emb_hash"]) == (rb["count"], rb["emb_hash"])


def test_out_of_core_partition_streaming_same_counts(small):
    """Out-of-core table builds that stream adjacency partitions (1 KiB each, so
    hub lists get partitions of their own) or read the mapped adjacency in place
    give the in-core counts and hashes, one query at a time and batched."""
    qs = [q for q in gem.gen_queries(small, 5, gem.ANY, 6, seed=6200)
          if oracle.count(small, q, want_hash=False, work_cap=100_000_000)[2]]
    opts = dict(time_cap_ms=30000, ooc=True, budget_bytes=2 << 30, ooc_part_kib=1)
    with gem.Context(time_cap_ms=30000) as a, gem.Context(ooc_stream=1, **opts) as b, \
            gem.Context(ooc_stream=2, **opts) as c:
        for x in (a, b, c):
            x.load_graph(small)
        st = b.ooc_stats()
        assert st["partitions"] > 16 and st["max_part_bytes"] > 1024  # some vertex list exceeds 1 KiB
        for q in qs:
            ra = a.run(q, mode=gem.MODE_HASH)
            for x in (b, c):
                rx = x.run(q, mode=gem.MODE_HASH)
                assert (rx["count"], rx["emb_hash"]) == (ra["count"], ra["emb_hash"])
        _, rs_a = a.batch(qs, mode=gem.MODE_HASH)
        _, rs_b = b.batch(qs, mode=gem.MODE_HASH)
        assert [(r["count"], r["emb_hash"]) for r in rs_b] == [(r["count"], r["emb_hash"]) for r in rs_a]
        sb, sc = b.ooc_stats(), c.ooc_stats()
        assert sb["waves_streamed"] >= len(qs) + 1 and sb["waves_in_place"] == 0
        assert sb["parts_streamed"] >= 2 * sb["waves_streamed"] and sb["bytes_streamed"] > 0
        assert sc["waves_streamed"] == 0 and sc["waves_in_place"] == len(qs) and sc["bytes_streamed"] == 0


def test_out_of_core_spills_tables_beyond_the_device_budget(small):
    """Out of core, a single query whose edge-table values do not fit the
    device budget keeps them in mapped pinned host memory: same count and
    hash as in core, and the spill is counted."""
    qs = [q for q in gem.gen_queries(small, 4, gem.ANY, 8, seed=6300)
          if oracle.count(small, q, want_hash=False, work_cap=100_000_000)[2]]
    with gem.Context(time_cap_ms=30000) as a:
        a.load_graph(small)
        runs = [(a.run(x, mode=gem.MODE_HASH), x) for x in qs]
    ra, q = max(runs, key=lambda t: t[0]["table_total"])  # the query with the largest tables
    with gem.Context(time_cap_ms=30000, ooc=True, budget_bytes=2 << 30) as b:
        b.load_graph(small)
        rb = b.run(q, mode=gem.MODE_HASH)
        resident = b.ooc_stats()["resident_bytes"]
    assert (rb["count"], rb["emb_hash"]) == (ra["count"], ra["emb_hash"])
    values = 4 * rb["table_total"]
    assert values >= 4096
    # a budget that holds everything of the wave but half of the values (the
    # context's own resident bytes decide whether the neighbourhood hash fits,
    # so the budget is settled on the resident bytes of a context that has it)
    budget = resident + rb["arena_bytes"] - values // 2
    for _ in range(3):
        with gem.Context(time_cap_ms=30000, ooc=True, budget_bytes=budget) as c:
            c.load_graph(small)
            res_c = c.ooc_stats()["resident_bytes"]
            if res_c + rb["arena_bytes"] - values // 2 != budget:
                budget = res_c + rb["arena_bytes"] - values // 2
                continue
            rc = c.run(q, mode=gem.MODE_HASH)
            st = c.ooc_stats()
            break
    assert (rc["count"], rc["emb_hash"]) == (ra["count"], ra["emb_hash"])
    assert st["waves_spilled"] == 1 and st["bytes_spilled"] >= values


def test_batch_splits_waves_under_a_tight_budget(small, gctx):
    """A wave whose tables exceed the device budget is split and retried: at the
    smallest budget that runs the batch, every result equals the plain run's and
    the batch took more than one wave."""
    qs = [q for k in (4, 5) for q in gem.gen_queries(small, k, gem.ANY, 40, seed=6300 + k)]
    plain = [gctx.run(q, mode=gem.MODE_HASH) for q in qs]
    assert all(p["status"] == "OK" for p in plain)
    _, one = gctx.batch(qs, mode=gem.MODE_HASH)
    assert len({r["wave"] for r in one}) == 1
    # budgets rise in 256 KiB steps: the first one that runs every query holds
    # the largest single query's wave but not the whole batch's
    found = None
    for kib in range(4096, 65536, 256):
        try:
            c = gem.Context(time_cap_ms=30000, budget_bytes=kib << 10)
            c.load_graph(small)
        except gem.GemError:
            continue
        with c:
            st, rs = c.batch(qs, mode=gem.MODE_HASH)
        if all(r["status"] == "OK" for r in rs):
            found = (kib, rs)
            break
        assert all(r["status"] in ("OK", "ERR_OOM") for r in rs)
    assert found is not None
    kib, rs = found
    assert [(r["count"], r["emb_hash"]) for r in rs] == [(p["count"], p["emb_hash"]) for p in plain]
    assert len({r["wave"] for r in rs}) > 1, kib


def test_autotune_keeps_results(small):
    qs = []
    for k in (3, 4, 6):
        for q in gem.gen_queries(small, k, gem.ANY, 4, seed=7000 + k):
            if oracle.count(small, q, want_hash=False, work_cap=100_000_000)[2]:
                qs.append(q)
    with gem.Context(time_cap_ms=30000) as c:
        c.load_graph(small)
        before = [c.run(q)["count"] for q in qs]
        rep = c.autotune(qs, trial_cap_ms=5000)
        assert rep and all(v["blocks_per_sm"] >= 1 and v["donate_max_level"] >= 1 for v in rep.values())
        st, after = c.batch(qs)
        assert st == 0 and [r["count"] for r in after] == before


REF_COUNTS = os.path.join(os.path.dirname(__file__), "golden", "ref_counts.json")


@pytest.mark.skipif(not os.path.exists(REF_COUNTS), reason="reference-binary fixture not generated")
def test_counts_match_reference_binary():
    """Counts printed by the reference's own in-core binary (a uint32 print,
    in-core/src/main.cu:233) equal the GPU count mod 2^32 on every recorded
    case, including those too large for the oracle's work cap."""
    with open(REF_COUNTS) as f:
        data = json.load(f)
    graphs, checked = {}, 0
    for c in data["cases"]:
        if c["exit"] != 0 or len(c["printed"]) != 1:
            continue
        gd = c["graph"]
        if gd["name"] not in graphs:
            g = gem.HostGraph.rmat(gd["scale"], gd["edge_factor"], seed=gd["seed"]).set_labels(
                gd["labels"], gd["zipf_s"], seed=gd["seed"] ^ 0x4C)
            ctx = gem.Context(time_cap_ms=60000)
            ctx.load_graph(g)
            graphs[gd["name"]] = ctx
        r = graphs[gd["name"]].run(gem.Query(c["labels"], c["edges"]))
        assert r["status"] == "OK"
        assert r["count"] % (1 << 32) == c["printed"][0], (gd["name"], c["labels"], c["edges"], r["count"])
        checked += 1
    for ctx in graphs.values():
        ctx.close()
    assert checked >= 10


def test_relaxed_counts_match_oracle(small, gctx):
    """gem_relaxed_run: every relaxed query's count equals the oracle's count
    of that query (each relaxed query is matched exactly)."""
    for k, dens, t in ((4, gem.DENSE, 2), (5, gem.ANY, 1), (6, gem.SPARSE, 1)):
        for q in gem.gen_queries(small, k, dens, 1, seed=300 + k):
            out = gctx.relaxed(q, t)
            assert [et for et, _ in out] == gem.relaxed_sets(q, t)
            for et, r in out:
                assert r["status"] == "OK", r
                exp, _, ok = oracle.count(small, gem.relaxed_query(q, et), want_hash=False)
                assert ok and r["count"] == exp, (q.edges.tolist(), bin(et), r["count"], exp)


REF_RELAXED = os.path.join(os.path.dirname(__file__), "golden", "ref_relaxed.json")


@pytest.mark.skipif(not os.path.exists(REF_RELAXED), reason="reference relaxed fixture not generated")
def test_relaxed_counts_match_reference_binary():
    """gem_relaxed_run at the reference's threshold returns the reference
    binary's relaxed queries with its printed counts (mod 2^32)."""
    with open(REF_RELAXED) as f:
        data = json.load(f)
    ctxs, checked = {}, 0
    for c in data["cases"]:
        if c["exit"] != 0 or not c["printed"]:
            continue
        gd = c["graph"]
        if gd["name"] not in ctxs:
            g = gem.HostGraph.rmat(gd["scale"], gd["edge_factor"], seed=gd["seed"]).set_labels(
                gd["labels"], gd["zipf_s"], seed=gd["seed"] ^ 0x4C)
            ctx = gem.Context(time_cap_ms=60000)
            ctx.load_graph(g)
            ctxs[gd["name"]] = ctx
        ref = {int(et, 2): cnt for et, cnt in zip(c["et"], c["printed"])}
        got = ctxs[gd["name"]].relaxed(gem.Query(c["labels"], c["edges"]), data["threshold"])
        assert {et for et, _ in got} == set(ref)
        for et, r in got:
            assert r["status"] == "OK" and r["count"] % (1 << 32) == ref[et], (c["edges"], bin(et), r["count"])
            checked += 1
    for ctx in ctxs.values():
        ctx.close()
    assert checked >= 20
