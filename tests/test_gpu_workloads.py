"""The benchmark's workloads on the GPU against the CPU oracle, bit-exact.

* Configuration 1 exactly as bench.py builds it (R-MAT scale 16, edge factor
  8, 8 uniform labels, the 100 random-walk 4-vertex queries): every query's
  count and embedding hash from one batch, and every plain count.
* The configuration-3 mix (query sizes 4 to 32, alternately sparse and
  dense) on a scale-10 graph with 16 Zipf labels, where the oracle finishes
  most of them: one batch in hash mode and one in count mode (closed-form
  suffixes), every query the oracle finishes compared.
* A batch under a time cap: the cheap queries of the wave finish exactly
  while an expensive one runs into the cap.
"""
import numpy as np
import pytest

import bench
import gem_b200 as gem
import oracle

pytestmark = pytest.mark.gpu


def test_config1_pool_matches_oracle():
    g, _ = bench.make_graph(gem, "rmat16")
    pool = bench.config1_pool(gem, g)
    assert len(pool) == 100
    with gem.Context(time_cap_ms=60000) as c:
        c.load_graph(g)
        st, rh = c.batch(pool, mode=gem.MODE_HASH)
        assert st == 0
        st, rc = c.batch(pool)
        assert st == 0
        plain = [c.run(q)["count"] for q in pool]
    for i, q in enumerate(pool):
        cnt, h, ok = oracle.count(g, q, want_hash=True)
        assert ok
        assert rh[i]["status"] == "OK" and rh[i]["count"] == cnt and rh[i]["emb_hash"] == h, i
        assert rc[i]["status"] == "OK" and rc[i]["count"] == cnt, i
        assert plain[i] == cnt, i


def test_mixed_size_batch_matches_oracle():
    g = gem.HostGraph.rmat(10, 8, seed=0x47454D0A).set_labels(16, 1.0, seed=0x47454D0A ^ 0x4C)
    pool = bench.mix_pool(gem, g, 120)
    assert {q.nv for q in pool} == set(bench.MIX_SIZES)
    # the queries the oracle finishes (under a work cap), all sizes, in one batch
    checked = []
    for q in pool:
        cnt, h, ok = oracle.count(g, q, want_hash=True, work_cap=100_000_000)
        if ok:
            checked.append((q, cnt, h))
    assert len(checked) >= 50 and {24, 32} <= {q.nv for q, _, _ in checked}, len(checked)
    qs = [q for q, _, _ in checked]
    with gem.Context(time_cap_ms=60000) as c:
        c.load_graph(g)
        st, rh = c.batch(qs, mode=gem.MODE_HASH)
        st2, rc = c.batch(qs)
    assert st == 0 and st2 == 0
    for i, (q, cnt, h) in enumerate(checked):
        assert rh[i]["status"] == "OK" and rh[i]["count"] == cnt and rh[i]["emb_hash"] == h, (i, q.nv)
        assert rc[i]["status"] == "OK" and rc[i]["count"] == cnt, (i, q.nv)


def test_capped_wave_keeps_cheap_queries_exact():
    g, _ = bench.make_graph(gem, "rmat16")
    cheap = bench.config1_pool(gem, g, 40)
    heavy = gem.gen_queries(g, 32, gem.SPARSE, 1, seed=0x5EA)
    qs = heavy + cheap  # the expensive query first in the batch
    with gem.Context(time_cap_ms=300) as c:
        c.load_graph(g)
        assert c.run(heavy[0], raise_on_error=False)["status"] == "ERR_TIMEOUT"
        _, rs = c.batch(qs)
    assert rs[0]["status"] == "ERR_TIMEOUT"
    for q, r in zip(cheap, rs[1:]):
        cnt, _, ok = oracle.count(g, q, want_hash=False)
        assert ok and r["status"] == "OK" and r["count"] == cnt


def test_two_lane_batch_matches_plain():
    """A batch of more query vertices than one wave takes runs its waves on
    two lanes (their joins beside the other lane's table builds): every count
    equals the plain run's and the oracle's, and waves of both lanes overlap
    on the device timeline."""
    g, _ = bench.make_graph(gem, "rmat16")
    pool = bench.config1_pool(gem, g)
    qs = pool * 12  # 4,800 query vertices: more than one wave
    expect = [oracle.count(g, q, want_hash=False)[0] for q in pool]
    with gem.Context(time_cap_ms=60000) as c:
        c.load_graph(g)
        for _ in range(2):  # the second batch reuses the lane
            st, rs = c.batch(qs)
            assert st == 0
            for i, r in enumerate(rs):
                assert r["status"] == "OK" and r["count"] == expect[i % len(pool)], i
        plain = [c.run(q)["count"] for q in pool]
    assert plain == expect
    iv = sorted({r["wave"]: (r["t_begin_ms"], r["t_end_ms"]) for r in rs}.values())
    assert len(iv) >= 2
    assert any(iv[b][0] < iv[a][1] for a in range(len(iv)) for b in range(a + 1, len(iv)))


def test_out_of_core_two_lane_batch_matches_in_core():
    """Out of core, a multi-wave batch runs on two lanes, each streaming the
    adjacency partitions through its own staging buffers (one lane's copies
    beside the other lane's join): same counts as in core, and the
    streaming counters cover both lanes."""
    g, _ = bench.make_graph(gem, "rmat16")
    pool = bench.config1_pool(gem, g)
    qs = pool * 12
    with gem.Context(time_cap_ms=60000) as a:
        a.load_graph(g)
        _, ra = a.batch(qs)
    with gem.Context(time_cap_ms=60000, ooc=True, ooc_stream=1, ooc_part_kib=64) as b:
        b.load_graph(g)
        _, rb = b.batch(qs)
        st = b.ooc_stats()
    assert [(r["status"], r["count"]) for r in rb] == [(r["status"], r["count"]) for r in ra]
    waves = {r["wave"] for r in rb}
    assert st["waves_streamed"] == len(waves) and st["bytes_streamed"] > 0


def _signatures(qs):
    """Filter-row signatures (label, degree, sorted neighbour labels) of the
    query vertices: a wave has one row per distinct signature."""
    sigs = set()
    for q in qs:
        nb = [[] for _ in range(q.nv)]
        for a, b in q.edges.tolist():
            nb[a].append(int(q.labels[b]))
            nb[b].append(int(q.labels[a]))
        for u in range(q.nv):
            sigs.add((int(q.labels[u]), len(nb[u]), tuple(sorted(nb[u]))))
    return sigs


def test_wave_with_many_sources_matches_oracle():
    """A wave with well over 1,024 distinct filter rows: the table passes
    find a vertex's sources in several 32-word chunks of its source column
    and stage target columns of more than 32 words.  Every count the oracle
    finishes equals the batch's."""
    g = gem.HostGraph.rmat(10, 8, seed=0x47454D0A).set_labels(16, 1.0, seed=0x47454D0A ^ 0x4C)
    pool = gem.gen_queries(g, 8, gem.SPARSE, 480, seed=0x5109)
    assert sum(q.nv for q in pool) <= 4096  # one wave's rows
    assert len(_signatures(pool)) >= 2000
    with gem.Context(time_cap_ms=20000) as c:
        c.load_graph(g)
        st, rb = c.batch(pool)
    assert len({r["wave"] for r in rb}) <= 2
    checked = 0
    for i, q in enumerate(pool):
        cnt, _, ok = oracle.count(g, q, want_hash=False, work_cap=20_000_000)
        if ok:
            assert rb[i]["status"] == "OK" and rb[i]["count"] == cnt, (i, rb[i]["status"])
            checked += 1
    assert checked >= 300, checked
