"""Runs the reference's own binaries on configuration 1's queries and records
the phase times they print, beside the counts (measurement infrastructure,
run on a GPU machine; the binaries come from oracle/ref/Makefile and
oracle/ref/Makefile.ooc).

Configuration 1: R-MAT scale 16, edge factor 8, 8 uniform labels, the
random-walk 4-vertex queries of seed 0x51000 (the benchmark's pool).  The
first N queries are written as the reference's text files (ascending vertex
lines, sorted edge lines) and run with threshold 0 (its default is 2):

* the out-of-core binary in directory mode (one child process per query,
  out-of-core/src/main.cu:334-410): `Filter time` and `construct time` are
  its host-side OpenMP filter and edge-table build
  (out-of-core/lib/filter/src/filter.cu:61-295,
  out-of-core/lib/structure/src/unifiedTrie.cu:1224-1427), `Join Time` its
  GPU join.  It pins (MemAvailable - 2 GiB) of host memory, capped by
  RLIMIT_MEMLOCK (out-of-core/lib/utils/src/cuda_helpers.cu:102-175): the
  run lowers that limit to PIN_GIB so the pinned pool stays bounded.
  OMP_NUM_THREADS is set to all host cores (without it the reference caps
  its filter at 16 and its table build at 4 threads);
* the in-core binary, one process per query: its `Filter time`, `Build Hash
  Table time`, `initVertexTries time`, `construct time` and `Join Time`
  (in-core/src/main.cu:145-227), all GPU phases; again with `-t 1`
  (relaxed matching, one count per relaxed query), beside this library's
  gem_relaxed_run on the same files (counts compared modulo 2^32), and at
  `-t 1` on 4-vertex queries with a cycle, which have relaxed queries.

The printed counts are checked against the oracle modulo 2^32 (both
binaries print them through a uint32_t).

Usage: python oracle/ref/time_reference.py <out.json> [n_queries] [work_dir]
"""
import json
import os
import re
import resource
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

PIN_GIB = 8
PHASES = ("Filter time", "Build Hash Table time", "initVertexTries time", "construct time")


def parse(text):
    """Per query (in print order): phase times in us, join time in us, counts."""
    out, cur = [], None
    for line in text.splitlines():
        m = re.match(r"^(Filter time|Build Hash Table time|initVertexTries time|construct time): (\d+) us", line)
        if m:
            if m.group(1) == "Filter time":
                cur = {"us": {}, "counts": []}
                out.append(cur)
            if cur is not None:
                cur["us"][m.group(1)] = int(m.group(2))
            continue
        m = re.match(r"^Join Time: (\d+) us", line)
        if m and cur is not None:
            cur["us"]["Join Time"] = int(m.group(1))
            continue
        m = re.match(r"^Relaxed Query ET ([01]+): (\d+) matches", line)
        if m and cur is not None:
            cur["counts"].append(int(m.group(2)))
    return out


def main():
    out_path = sys.argv[1]
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 8
    work = sys.argv[3] if len(sys.argv) > 3 else os.path.join(os.path.dirname(out_path), "ref_timing_inputs")
    os.makedirs(os.path.join(work, "queries"), exist_ok=True)
    g = oracle.set_labels(oracle.rmat(16, 8, seed=0x47454D00 + 16), 8, 0.0, seed=(0x47454D00 + 16) ^ 0x4C)
    qs = oracle.gen_queries(g, 4, 0, 100, seed=0x51000)[:n]
    gpath = os.path.join(work, "rmat16.graph")
    write_graph(g, gpath)
    for i, q in enumerate(qs):
        write_query(q, os.path.join(work, "queries", f"Q_{i}.in"))
    expect = [oracle.count(g, q, want_hash=False)[0] % (1 << 32) for q in qs]
    ncores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(ncores))
    res = {"workload": "rmat16-ef8-uniform8, first %d queries of the pool" % n, "host_cores": ncores,
           "pinned_cap_gib": PIN_GIB, "expect_mod_2_32": expect}

    def limit_pinned():
        resource.setrlimit(resource.RLIMIT_MEMLOCK, (PIN_GIB << 30, PIN_GIB << 30))

    ooc = os.path.join(ROOT, "oracle", "_ref", "GEM_ooc")
    t0 = time.time()
    r = subprocess.run([ooc, "-q", os.path.join(work, "queries"), "-d", gpath, "-t", "0"], capture_output=True,
                       text=True, env=env, preexec_fn=limit_pinned, timeout=1800)
    res["out_of_core"] = {"exit": r.returncode, "wall_s": round(time.time() - t0, 1), "queries": parse(r.stdout),
                          "summary": [l for l in r.stdout.splitlines() if l.startswith(("success=", "[failed]"))],
                          "stderr_tail": r.stderr[-400:]}
    ic = os.path.join(ROOT, "oracle", "_ref", "GEM_ic")
    runs = []
    for i in range(n):
        t0 = time.time()
        r = subprocess.run([ic, "-q", os.path.join(work, "queries", f"Q_{i}.in"), "-d", gpath, "-t", "0", "-g", "0"],
                           capture_output=True, text=True, env=env, timeout=600)
        p = parse(r.stdout)
        runs.append({"exit": r.returncode, "wall_s": round(time.time() - t0, 1), **(p[0] if p else {})})
    res["in_core"] = runs
    # relaxed matching (-t 1): the in-core binary's phase times and its
    # per-relaxed-query counts, beside gem_relaxed_run's on the same queries
    rel = []
    for i in range(n):
        t0 = time.time()
        r = subprocess.run([ic, "-q", os.path.join(work, "queries", f"Q_{i}.in"), "-d", gpath, "-t", "1", "-g", "0"],
                           capture_output=True, text=True, env=env, timeout=600)
        p = parse(r.stdout)
        rel.append({"exit": r.returncode, "wall_s": round(time.time() - t0, 1), **(p[0] if p else {})})
    res["in_core_t1"] = rel
    try:
        import gem_b200 as gem
        gg = gem.HostGraph.read_text(gpath)
        with gem.Context() as c:
            c.load_graph(gg)
            ours = []
            for i in range(n):
                q = gem.Query.read_text(os.path.join(work, "queries", f"Q_{i}.in"))
                c.relaxed(q, 1)
                t0 = time.time()
                out = c.relaxed(q, 1)
                ours.append({"wall_ms": round((time.time() - t0) * 1e3, 3),
                             "device_ms": round(sum({r["wave"]: r["ms"]["total"] for _, r in out}.values()), 3),
                             "counts_mod_2_32": sorted(r["count"] % (1 << 32) for _, r in out)})
        res["gem_t1"] = ours
        res["t1_counts_equal"] = sum(1 for a, b in zip(rel, ours) if sorted(a.get("counts", [])) == b["counts_mod_2_32"])
    except Exception as e:  # the library is optional here: the reference's figures stand alone
        res["gem_t1_error"] = str(e)[:200]
    res["relaxed_dense"] = relaxed_dense(g, gpath, work, env, ic)
    ok = [q["counts"] == [e] for q, e in zip(res["out_of_core"]["queries"], expect)]
    res["out_of_core"]["counts_equal_oracle"] = sum(ok)
    res["in_core_counts_equal_oracle"] = sum(1 for q, e in zip(runs, expect) if q.get("counts") == [e])
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps({k: v for k, v in res.items() if k not in ("in_core",)})[:3000])


def relaxed_t1(q):
    """Edge sets of q's relaxed queries at threshold 1 (bit j: q's edge j kept):
    q itself and q without one edge, where the rest still connects q."""
    e = [tuple(x) for x in q.edges.reshape(-1, 2).tolist()]
    full = (1 << len(e)) - 1
    out = [full]
    if len(e) + 1 > q.nv:  # not a spanning tree: an edge can go
        for j in range(len(e)):
            keep = [e[i] for i in range(len(e)) if i != j]
            seen, todo = {0}, [0]
            while todo:
                u = todo.pop()
                for a, b in keep:
                    for x, y in ((a, b), (b, a)):
                        if x == u and y not in seen:
                            seen.add(y)
                            todo.append(y)
            if len(seen) == q.nv:
                out.append(full & ~(1 << j))
    return out


def relaxed_dense(g, gpath, work, env, ic, n=6):
    """Relaxed matching (-t 1) on 4-vertex queries with a cycle, which have
    relaxed queries (a tree has none): the in-core binary against
    gem_relaxed_run, counts compared modulo 2^32.  Only queries whose relaxed
    counts (by the oracle) stay at most 2e8 are run, the size of the
    configuration-1 counts the reference handled here."""
    picked = []
    for q in oracle.gen_queries(g, 4, 2, 60, seed=0x51100):
        ne = len(q.edges.reshape(-1, 2))
        if ne < 4 or ne > 5:
            continue
        counts = []
        for m in relaxed_t1(q):
            ed = [x for j, x in enumerate(q.edges.reshape(-1, 2).tolist()) if (m >> j) & 1]
            c, _, ok = oracle.count(g, oracle.Query(q.labels, ed), want_hash=False, work_cap=2_000_000_000)
            if not ok or c > 200_000_000:
                counts = None
                break
            counts.append(c % (1 << 32))
        if counts:
            picked.append((q, sorted(counts)))
        if len(picked) == n:
            break
    out = {"queries": len(picked), "relaxed_per_query": [len(c) for _, c in picked], "reference": [], "gem": []}
    for i, (q, _) in enumerate(picked):
        qpath = os.path.join(work, "queries_relaxed", f"R_{i}.in")
        os.makedirs(os.path.dirname(qpath), exist_ok=True)
        write_query(q, qpath)
        t0 = time.time()
        r = subprocess.run([ic, "-q", qpath, "-d", gpath, "-t", "1", "-g", "0"], capture_output=True, text=True,
                           env=env, timeout=600)
        p = parse(r.stdout)
        out["reference"].append({"exit": r.returncode, "wall_s": round(time.time() - t0, 1), **(p[0] if p else {})})
    try:
        import gem_b200 as gem
        with gem.Context() as c:
            c.load_graph(gem.HostGraph.read_text(gpath))
            for i in range(len(picked)):
                q = gem.Query.read_text(os.path.join(work, "queries_relaxed", f"R_{i}.in"))
                c.relaxed(q, 1)
                t0 = time.time()
                res = c.relaxed(q, 1)
                out["gem"].append({"wall_ms": round((time.time() - t0) * 1e3, 3),
                                   "device_ms": round(sum({r["wave"]: r["ms"]["total"] for _, r in res}.values()), 3),
                                   "counts_mod_2_32": sorted(r["count"] % (1 << 32) for _, r in res)})
    except Exception as e:  # the library is optional here: the reference's figures stand alone
        out["gem_error"] = str(e)[:200]
    out["oracle_equal_reference"] = sum(1 for (_, c), r in zip(picked, out["reference"])
                                        if sorted(r.get("counts", [])) == c)
    out["gem_equal_reference"] = sum(1 for a, b in zip(out["reference"], out["gem"])
                                     if sorted(a.get("counts", [])) == b["counts_mod_2_32"])
    return out


def write_graph(g, path):
    off, nbr, lab = g.arrays()
    with open(path, "w") as f:
        nv = len(lab)
        ne = int(off[-1]) // 2
        f.write(f"t {nv} {ne}\n")
        for v in range(nv):
            f.write(f"v {v} {int(lab[v])} {int(off[v + 1] - off[v])}\n")
        for v in range(nv):
            for w in nbr[off[v]:off[v + 1]]:
                if w > v:
                    f.write(f"e {v} {int(w)}\n")


def write_query(q, path):
    deg = [0] * q.nv
    for a, b in q.edges.tolist():
        deg[a] += 1
        deg[b] += 1
    with open(path, "w") as f:
        f.write(f"t {q.nv} {q.ne}\n")
        for u in range(q.nv):
            f.write(f"v {u} {int(q.labels[u])} {deg[u]}\n")
        for a, b in sorted(tuple(sorted(e)) for e in q.edges.tolist()):
            f.write(f"e {a} {b}\n")


if __name__ == "__main__":
    main()
