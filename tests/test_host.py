"""Host-side logic of libgem: ABI exports, generators, text IO, validation.
No device calls."""
import ctypes
import os
import re

import numpy as np
import pytest

import gem_b200 as gem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gem.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gem_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(gem.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(gem.EXPORTS)


def test_strerror():
    L = gem.lib()
    assert L.gem_strerror(0) == b"ok"
    assert b"time" in L.gem_strerror(4)


def test_rmat_deterministic_and_valid():
    a = gem.HostGraph.rmat(12, 8, seed=99)
    b = gem.HostGraph.rmat(12, 8, seed=99)
    c = gem.HostGraph.rmat(12, 8, seed=100)
    oa, na, _ = a.arrays()
    ob, nb, _ = b.arrays()
    oc, nc, _ = c.arrays()
    assert np.array_equal(oa, ob) and np.array_equal(na, nb)
    assert not (len(nc) == len(na) and np.array_equal(nc, na))
    # sorted, no self loops, symmetric
    for v in range(len(oa) - 1):
        lst = na[oa[v]:oa[v + 1]]
        assert np.all(np.diff(lst.astype(np.int64)) > 0)
        assert v not in lst
    src = np.repeat(np.arange(len(oa) - 1), np.diff(oa).astype(np.int64))
    fwd = set(zip(src.tolist(), na.tolist()))
    assert all((d, s) in fwd for s, d in list(fwd)[:5000])
    # edge count close to the sampled count minus duplicates
    assert 0.5 * 8 * 4096 * 2 < len(na) <= 8 * 4096 * 2


def test_labels_uniform_and_zipf():
    g = gem.HostGraph.rmat(14, 4, seed=5)
    g.set_labels(8, 0.0, seed=1)
    lab = g.arrays()[2]
    h = np.bincount(lab, minlength=8) / len(lab)
    assert np.all(np.abs(h - 1 / 8) < 0.02)
    g.set_labels(16, 1.0, seed=1)
    lab = g.arrays()[2]
    h = np.bincount(lab, minlength=16) / len(lab)
    expect = 1 / np.arange(1, 17)
    expect /= expect.sum()
    assert np.all(np.abs(h - expect) < 0.02)


def test_text_roundtrip(tmp_path):
    g = gem.HostGraph.rmat(9, 4, seed=2).set_labels(5, seed=3)
    p = str(tmp_path / "g.graph")
    g.write_text(p)
    g2 = gem.HostGraph.read_text(p)
    for x, y in zip(g.arrays(), g2.arrays()):
        assert np.array_equal(x, y)


def test_text_reader_accepts_unsorted_and_rejects_bad(tmp_path):
    p = tmp_path / "u.graph"
    p.write_text("t 3 2\nv 2 7 1\nv 0 5 1\nv 1 6 2\ne 2 1\ne 1 0\n")
    g = gem.HostGraph.read_text(str(p))
    off, nbr, lab = g.arrays()
    assert off.tolist() == [0, 1, 3, 4] and nbr.tolist() == [1, 0, 2, 1] and lab.tolist() == [5, 6, 7]
    bad = tmp_path / "b.graph"
    bad.write_text("t 3 2\nv 0 5 1\nv 1 6 1\nv 2 7 1\ne 2 1\ne 1 0\n")  # degree of 1 is 2
    with pytest.raises(gem.GemError):
        gem.HostGraph.read_text(str(bad))
    with pytest.raises(gem.GemError):
        gem.HostGraph.read_text(str(tmp_path / "missing.graph"))


def test_query_text_roundtrip(tmp_path):
    q = gem.Query([3, 1, 3, 2], [(0, 1), (1, 2), (2, 3), (3, 0)])
    p = str(tmp_path / "Q_0.in")
    q.write_text(p)
    q2 = gem.Query.read_text(p)
    assert q2.labels.tolist() == q.labels.tolist() and q2.edges.tolist() == q.edges.tolist()


@pytest.mark.parametrize("k,dens", [(4, gem.ANY), (8, gem.SPARSE), (8, gem.DENSE), (16, gem.SPARSE), (12, gem.DENSE)])
def test_random_walk_queries(k, dens):
    g = gem.HostGraph.rmat(12, 16, seed=4).set_labels(4, seed=4)
    qs = gem.gen_queries(g, k, dens, 12, seed=77)
    off, nbr, lab = g.arrays()
    for q in qs:
        assert q.nv == k
        adj = {u: set() for u in range(k)}
        for a, b in q.edges.tolist():
            adj[a].add(b)
            adj[b].add(a)
        seen, st = {0}, [0]
        while st:
            x = st.pop()
            for y in adj[x]:
                if y not in seen:
                    seen.add(y)
                    st.append(y)
        assert len(seen) == k
        avg = 2 * q.ne / k
        if dens == gem.SPARSE:
            assert avg <= 3
        if dens == gem.DENSE:
            assert avg > 3
    qs2 = gem.gen_queries(g, k, dens, 12, seed=77)
    assert all(np.array_equal(a.edges, b.edges) and np.array_equal(a.labels, b.labels) for a, b in zip(qs, qs2))


def _relaxed_py(q, threshold):
    """Independent enumeration: edge subsets with at most `threshold` edges
    removed whose edges connect all query vertices."""
    import itertools
    ne, nv = q.ne, q.nv
    edges = q.edges.tolist()
    out = set()
    for r in range(0, min(threshold, ne) + 1):
        for removed in itertools.combinations(range(ne), r):
            keep = [j for j in range(ne) if j not in removed]
            adj = {u: set() for u in range(nv)}
            for j in keep:
                a, b = edges[j]
                adj[a].add(b)
                adj[b].add(a)
            seen, stack = {0}, [0]
            while stack:
                u = stack.pop()
                for w in adj[u] - seen:
                    seen.add(w)
                    stack.append(w)
            if len(seen) == nv:
                out.add(sum(1 << j for j in keep))
    return out


def test_relaxed_sets_match_enumeration():
    """gem_relaxed_sets: the connected spanning edge subsets with at most T
    edges removed, fewest removed first (in-core/lib/plan/src/relax.cpp:84-142)."""
    qs = [gem.Query([0, 0, 0, 0], [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2)]),
          gem.Query([1, 2, 1], [(0, 1), (1, 2), (0, 2)]),
          gem.Query([0, 1, 2, 3], [(0, 1), (1, 2), (2, 3)]),
          gem.Query([0] * 5, [(i, j) for i in range(5) for j in range(i + 1, 5)]),
          gem.Query([3], [])]
    g = gem.HostGraph.rmat(10, 8, seed=7).set_labels(3, seed=8)
    qs += gem.gen_queries(g, 6, gem.DENSE, 4, seed=9) + gem.gen_queries(g, 8, gem.ANY, 4, seed=10)
    for q in qs:
        for t in (0, 1, 2, 3):
            got = gem.relaxed_sets(q, t)
            assert set(got) == _relaxed_py(q, t), (q.edges.tolist(), t)
            assert len(got) == len(set(got))
            removed = [q.ne - bin(x).count("1") for x in got]
            assert removed == sorted(removed) and (not got or got[0] == (1 << q.ne) - 1)


def test_relaxed_sets_cap():
    q = gem.Query([0] * 5, [(i, j) for i in range(5) for j in range(i + 1, 5)])
    n = len(gem.relaxed_sets(q, 3))
    with pytest.raises(gem.GemError):
        gem.relaxed_sets(q, 3, cap=n - 1)


# ---------------------------------------------------------------------------
# Planner (gem_plan_query), against a restatement of its rules: the closed-form
# suffix is an independent set chosen greedily (lowest degree, then most
# candidates, then lowest id) whose removal leaves the rest connected, with at
# most 4 suffix vertices per label, at most 16 labels and at most 32 backward
# lists per label group; the root has the fewest candidates per incident edge;
# each later level has the most matched neighbours, non-leaves first, then
# fewest candidates, highest degree, lowest id; suffix levels follow, by label.
# ---------------------------------------------------------------------------
def _plan_model(q, cnt, closed_form):
    n = q.nv
    adj = [0] * n
    for a, b in q.edges.tolist():
        adj[a] |= 1 << b
        adj[b] |= 1 << a
    deg = [bin(x).count("1") for x in adj]
    lab = [int(x) for x in q.labels]

    def connected_without(rem):
        alive = ((1 << n) - 1) & ~rem
        if not alive:
            return False
        seen = alive & -alive
        frontier = seen
        while frontier:
            nxt = 0
            for u in range(n):
                if frontier >> u & 1:
                    nxt |= adj[u]
            nxt &= alive & ~seen
            seen |= nxt
            frontier = nxt
        return seen == alive

    S = 0
    if closed_form and n >= 2:
        for u in sorted(range(n), key=lambda u: (deg[u], -int(cnt[u]), u)):
            if adj[u] & S:
                continue
            S2 = S | 1 << u
            if not connected_without(S2):
                continue
            members = [w for w in range(n) if S2 >> w & 1]
            same = [w for w in members if lab[w] == lab[u]]
            nback = deg[u] + sum(deg[w] for w in same if w != u)
            if len(same) > 4 or nback > 32 or len({lab[w] for w in members}) > 16:
                continue
            S = S2
    nenum = n - bin(S).count("1")
    used, order = 0, []
    for k in range(nenum):
        best = None
        for u in range(n):
            if (used | S) >> u & 1:
                continue
            back = bin(adj[u] & used).count("1")
            if k > 0 and back == 0:
                continue
            d = deg[u]
            key = (int(int(cnt[u]) / (d + 1) * 1024.0), -d, u) if k == 0 else (-back, 1 if d <= 1 else 0, int(cnt[u]), -d, u)
            if best is None or key < best[0]:
                best = (key, u)
        order.append(best[1])
        used |= 1 << best[1]
    suffix = sorted((u for u in range(n) if S >> u & 1), key=lambda u: (lab[u], u))
    return nenum, order + suffix, adj


@pytest.mark.parametrize("closed_form", [True, False])
def test_planner_matches_its_rules(closed_form):
    g = gem.HostGraph.rmat(12, 8, seed=11).set_labels(3, seed=12)
    rng = np.random.default_rng(5)
    n_checked = 0
    for k, dens in ((3, gem.ANY), (4, gem.ANY), (5, gem.SPARSE), (6, gem.DENSE), (8, gem.ANY), (12, gem.SPARSE),
                    (16, gem.DENSE), (32, gem.SPARSE)):
        for q in gem.gen_queries(g, k, dens, 6, seed=700 + k):
            cnt = rng.integers(1, 5000, size=q.nv)
            ne, order = gem.plan(q, cnt, closed_form)
            exp_ne, exp_order, adj = _plan_model(q, cnt, closed_form)
            assert (ne, order) == (exp_ne, exp_order), (q.labels.tolist(), q.edges.tolist(), cnt.tolist())
            # structure: a permutation; the prefix grows connected; the suffix is independent
            assert sorted(order) == list(range(q.nv))
            seen = 1 << order[0]
            for u in order[1:ne]:
                assert adj[u] & seen
                seen |= 1 << u
            suf = order[ne:]
            assert all(not (adj[u] >> v & 1) for u in suf for v in suf)
            if not closed_form:
                assert ne == q.nv
            n_checked += 1
    assert n_checked >= 40


def test_planner_rejects_bad_input():
    q = gem.Query([0, 1, 2], [(0, 1)])  # disconnected
    with pytest.raises(gem.GemError):
        gem.plan(q, [5, 5, 5])
    with pytest.raises(ValueError):
        gem.plan(gem.Query([0, 1], [(0, 1)]), [5])


@pytest.mark.parametrize("part_kib", [1, 4, 64])
def test_out_of_core_partitions(part_kib):
    """Partition bounds (gem_hgraph_partitions): consecutive vertex ranges that
    cover every vertex, each of at most part_kib KiB of arcs unless it holds a
    single vertex whose list is longer, and each as long as the bound allows."""
    g = gem.HostGraph.rmat(12, 8, seed=21).set_labels(3, seed=22)
    off, _, _ = g.arrays()
    cap = (part_kib << 10) // 4
    pv = g.partitions(part_kib)
    assert pv[0] == 0 and pv[-1] == g.nv and np.all(np.diff(pv.astype(np.int64)) > 0)
    big = 0
    for a, b in zip(pv[:-1].tolist(), pv[1:].tolist()):
        arcs = int(off[b] - off[a])
        if b - a == 1 and arcs > cap:
            big += 1  # a hub list longer than a partition: alone
        else:
            assert arcs <= cap
        if b < g.nv:
            assert int(off[b + 1] - off[a]) > cap  # one more vertex would not fit
    if part_kib == 1:
        assert big > 0  # this graph has lists longer than 256 arcs
    assert len(g.partitions(0)) == 2  # the default 16 MiB holds the whole graph
