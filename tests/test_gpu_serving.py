"""Serving (gem_submit / gem_poll) on the GPU.

* Two serving lanes: waves formed while another wave is on the device run at
  the same time (their device intervals, from CUDA events on one timeline,
  intersect), and every result equals the query's count alone (plain) and
  the CPU oracle's.
* Admission: the bytes gem_submit reserves for a query bound what its wave
  takes from the device arena, without a needlessly large margin.
"""
import time

import numpy as np
import pytest

import bench
import gem_b200 as gem
import oracle

pytestmark = pytest.mark.gpu


def test_serving_lanes_overlap_and_match_oracle():
    g, _ = bench.make_graph(gem, "rmat16")
    pool = bench.config1_pool(gem, g)
    expect = [oracle.count(g, q, want_hash=False)[0] for q in pool]
    qs = pool * 4
    with gem.Context(time_cap_ms=60000) as c:
        c.load_graph(g)
        alone = [c.run(q)["count"] for q in pool]
        assert alone == expect
    with gem.Context(time_cap_ms=60000) as c:
        c.load_graph(g)
        tickets = []
        for k in range(0, len(qs), 25):  # arrivals in groups, none waiting for results
            tickets += [c.submit(q) for q in qs[k:k + 25]]
        assert all(t is not None for t in tickets)
        res, t0 = {}, time.time()
        while len(res) < len(tickets):
            assert time.time() - t0 < 120
            for i, t in enumerate(tickets):
                if i not in res:
                    r = c.poll(t)
                    if r is not None:
                        res[i] = r
    for i, q in enumerate(qs):
        assert res[i]["status"] == "OK" and res[i]["count"] == expect[i % len(pool)], i
    waves = {}
    for r in res.values():
        waves[r["wave"]] = (r["t_begin_ms"], r["t_end_ms"])
    iv = sorted(waves.values())
    assert len(iv) >= 2
    overlapping = sum(1 for a in range(len(iv)) for b in range(a + 1, len(iv))
                      if iv[b][0] < iv[a][1] and iv[a][0] < iv[b][1])
    assert overlapping >= 1, iv


def test_admission_estimate_bounds_wave_bytes():
    ratios = []
    for g in (bench.make_graph(gem, "rmat16")[0],
              gem.HostGraph.rmat(12, 8, seed=0x47454D0C).set_labels(16, 1.0, seed=0x47454D0C ^ 0x4C)):
        qs = bench.config1_pool(gem, g, 40) + bench.mix_pool(gem, g, 60)
        with gem.Context(time_cap_ms=2000) as c:
            c.load_graph(g)
            for q in qs:
                est = c.estimate_bytes(q)
                r = c.run(q, raise_on_error=False)
                if r["arena_bytes"]:
                    assert r["arena_bytes"] <= est, (q.nv, q.ne, r["arena_bytes"], est)
                    ratios.append(est / r["arena_bytes"])
    assert len(ratios) >= 150
    assert float(np.median(ratios)) < 16.0, float(np.median(ratios))

