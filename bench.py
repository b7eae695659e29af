#!/usr/bin/env python3
"""Benchmark: exact subgraph-matching throughput on one B200 (queries/s and
embeddings/s, batched vs plain, p50/p99 latency).

Headline workload (default `rmat16`, the configuration whose every query
completes exactly): R-MAT scale 16 (65,536 vertices), edge factor 8,
(a,b,c,d) = (0.57,0.19,0.19,0.05), self loops and duplicates removed, uint32
CSR with sorted adjacency, 8 uniform labels; 100 random-walk queries of 4
vertices (seeded synthetic stand-ins; the reference's datasets are not used).
A step is one gem_batch_run over the 100 queries (one persistent join launch
per wave); `plain` runs the same queries one gem_query_run each.

The scale-22 workload (`--workload rmat22`: 4,194,304 vertices, edge factor
16, 16 labels Zipf(s=1.0), query sets 8 sparse / 8 dense / 16 sparse / 16
dense) is reported in the `rmat22` section: its random-walk queries have
10^13 to 10^17 embeddings each, so no exact method finishes them in a
bounded step; the section reports, per query under a device time cap,
whether it completed and the enumeration rate.  A query that exceeds the cap
is reported as capped, never as an exact count.

Its `out_of_core` part runs one batch of 4-vertex queries on that graph in
core, out of core with the adjacency streamed in partitions, and out of core
reading the pinned adjacency in place, and reports each mode's table-build
and wave times with equal counts.

The `serving` section submits the headline queries one by one through
gem_submit / gem_poll under Poisson arrivals (1,000 / 5,000 / 20,000 per
second, one second each) and reports latency percentiles and the achieved
rate; every result is checked against the batched count.

`value` is device-timed (CUDA events around each batch, inputs resident in
HBM), `e2e` is wall time around the C-ABI call from host buffers (query
arrays in, results out).  L2 is flushed between steps (a 256 MiB write).
With torchrun (N > 1) every rank runs an independent replica on its own share
of the batches (the path has no exchange step); rank 0 reports the max time.
`--impl reference` times the CPU restatement of the path (the reference has no
CPU join) on the host cores with all threads.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SETS = ((8, 1), (8, 2), (16, 1), (16, 2))  # (k, density: 1 sparse, 2 dense)
METRIC = "queries/s & embeddings/s on 1 B200, batched vs plain, exact counts; p50/p99 ms"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def batch_indices(step, rank, world, batch, pool_len):
    """Pool indices of one rank's batch at a step: the ranks of a step take
    consecutive batches of the cycled pool (weak scaling, no shared query)."""
    i = (step * world + rank) * batch
    return [(i + j) % pool_len for j in range(batch)]


def reduce_over_ranks(dist, tdev, twall, exact, emb, capped, e2e_exact):
    """Whole-job figures: the slowest rank's device and wall times, the sums of
    the per-rank counts (every rank calls this, in the same order)."""
    import torch
    t = torch.tensor([tdev, twall, float(exact), float(emb), float(capped), float(e2e_exact)], dtype=torch.float64)
    mx = t[:2].clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t[2:].clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(mx[1]), int(sm[0]), int(sm[1]), int(sm[2]), int(sm[3])


class Clocks:
    """nvidia-smi sampler during the timed region."""

    def __init__(self, gpu):
        self.gpu, self.samples, self.p = gpu, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def parse_sets(spec):
    """'8s,8d,16s,16d' -> ((8, 1), (8, 2), (16, 1), (16, 2)); a = any density."""
    out = []
    for tok in spec.split(","):
        tok = tok.strip()
        out.append((int(tok[:-1]), {"a": 0, "s": 1, "d": 2}[tok[-1]]))
    return tuple(out)


def make_workload(gem, name, sets_spec=None):
    if name == "rmat22":
        t = time.time()
        g = gem.HostGraph.rmat(22, 16, seed=0x47454D00 + 22).set_labels(16, 1.0, seed=(0x47454D00 + 22) ^ 0x4C)
        gen_s = time.time() - t
        desc = {"workload": "rmat22-ef16-zipf16", "scale": 22, "edge_factor": 16, "labels": 16, "zipf_s": 1.0}
        sets = SETS
    elif name == "rmat16":
        t = time.time()
        g = gem.HostGraph.rmat(16, 8, seed=0x47454D00 + 16).set_labels(8, 0.0, seed=(0x47454D00 + 16) ^ 0x4C)
        gen_s = time.time() - t
        desc = {"workload": "rmat16-ef8-uniform8", "scale": 16, "edge_factor": 8, "labels": 8, "zipf_s": 0.0}
        sets = ((4, 0),)
    else:
        raise SystemExit(f"unknown workload {name}")
    if sets_spec:
        sets = parse_sets(sets_spec)
    return g, desc, sets, gen_s


def query_pool(gem, g, sets, per_set):
    pools = [gem.gen_queries(g, k, d, per_set, seed=0x51000 + i) for i, (k, d) in enumerate(sets)]
    out = []
    for j in range(per_set):
        for p in pools:
            out.append(p[j])
    return out


def flush_l2(torch_dev):
    import torch
    buf = torch.empty(256 << 20, dtype=torch.uint8, device=torch_dev)
    buf.fill_(1)
    torch.cuda.synchronize()


def pctl(xs, p):
    if not xs:
        return None
    xs = sorted(xs)
    k = min(len(xs) - 1, max(0, int(round(p / 100.0 * (len(xs) - 1)))))
    return xs[k]


def run_gem(args):
    import gem_b200 as gem
    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    g, desc, sets, gen_s = make_workload(gem, args.workload, args.sets)
    pool = query_pool(gem, g, sets, args.per_set)
    B = args.batch
    ctx = gem.Context(device=local, time_cap_ms=args.cap_ms)
    ctx.load_graph(g)
    # the tuner runs the timed batch's queries (untimed); a wave's join lasts as long
    # as its heaviest query, so a sample without it tunes for the wrong critical path
    tuned = ctx.autotune(pool[: min(len(pool), args.batch)], trial_cap_ms=args.cap_ms) if args.autotune else {}

    def batch_of(step):
        return [pool[i] for i in batch_indices(step, rank, world, B, len(pool))]

    # warm-up (compiles nothing; touches code paths and the arena)
    for s in range(args.warmup):
        ctx.batch(batch_of(s))
    steps = list(range(args.warmup, args.warmup + args.steps))
    dev_ms, wall_ms, res_all = [], [], []
    h2d = d2h = launches = jbytes = n_joins = 0
    jms = 0.0
    phase = {"filter": 0.0, "tables": 0.0, "index": 0.0, "join": 0.0}
    with Clocks(local) as clk:
        for s in steps:
            qs = batch_of(s)
            flush_l2(dev)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            st, rs = ctx.batch(qs)
            torch.cuda.synchronize()
            # device time of the batch: sum over its waves (first kernel .. last kernel, CUDA events)
            waves = {}
            for r in rs:
                waves.setdefault(r["wave"], r)
            dev_ms.append(sum(r["ms"]["total"] for r in waves.values()))
            launches += sum(r["launches"] for r in waves.values())
            jbytes += sum(r["bytes_alg"][3] for r in waves.values())
            n_joins += len(waves)
            jms += sum(r["ms"]["join"] for r in waves.values())
            for k in phase:
                phase[k] += sum(r["ms"][k] for r in waves.values())
            res_all.append(rs)
    # end to end through the public API: query arrays in host memory, the
    # counts and statuses read back, timed on the host (a separate pass over
    # the same steps, so the device-timed pass keeps its per-wave records)
    e2e_same, e2e_exact = True, 0
    for i, s in enumerate(steps):
        qs = batch_of(s)
        flush_l2(dev)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, counts, status = ctx.batch_counts(qs)
        torch.cuda.synchronize()
        wall_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_same &= all(int(c) == r["count"] for c, r in zip(counts, res_all[i]) if r["status"] == "OK")
        e2e_exact += int((status == 0).sum())
        h2d += sum(4 * q.nv + 8 * q.ne for q in qs)  # the queries' label and edge arrays
        d2h += 64 * len(qs) + 1024  # per-query counters and the control block
    exact = sum(1 for rs in res_all for r in rs if r["status"] == "OK")
    capped = sum(1 for rs in res_all for r in rs if r["status"] == "ERR_TIMEOUT")
    emb = sum(r["count"] for rs in res_all for r in rs if r["status"] == "OK")
    tdev = sum(dev_ms) / 1e3
    twall = sum(wall_ms) / 1e3
    # join-kernel roofline from the batches' algorithmic bytes and join times
    jb = jbytes
    jt = jms / 1e3
    if dist:
        tdev, twall, exact, emb, capped, e2e_exact = reduce_over_ranks(dist, tdev, twall, exact, emb, capped, e2e_exact)
    # plain mode: the same queries, one gem_query_run each (rank 0)
    plain = {}
    if rank == 0 and args.plain > 0:
        lat, pe, pn, pdev = [], 0, 0, 0.0
        qs = batch_of(args.warmup)[: args.plain]
        same = True
        for q, rb in zip(qs, res_all[0]):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = ctx.run(q, raise_on_error=False)
            torch.cuda.synchronize()
            lat.append((time.perf_counter() - t0) * 1e3)
            pdev += r["ms"]["total"] / 1e3
            if r["status"] == "OK":
                pn += 1
                pe += r["count"]
                same &= rb["status"] != "OK" or rb["count"] == r["count"]
        plain = {"queries": len(lat), "exact": pn, "queries_per_s": pn / pdev if pdev else None,
                 "queries_per_s_wall": pn / (sum(lat) / 1e3) if lat else None,
                 "p50_ms": pctl(lat, 50), "p99_ms": pctl(lat, 99), "counts_equal_batched": same}
    ctx.close()
    serving = None
    if rank == 0 and args.serve_seconds > 0:
        ref = {i: r["count"] for i, r in enumerate(res_all[0])} if len(batch_of(args.warmup)) == len(pool) else {}
        serving = serving_section(gem, args, local, g, pool, ref) if ref else None
    c2 = None
    if rank == 0 and (args.c2_sample > 0 or args.ooc_sample > 0):
        t = time.time()
        g22 = gem.HostGraph.rmat(22, 16, seed=0x47454D00 + 22).set_labels(16, 1.0, seed=(0x47454D00 + 22) ^ 0x4C)
        gen22 = time.time() - t
        c2 = rmat22_section(gem, args, local, g22, gen22) if args.c2_sample > 0 else {"graph_gen_s": round(gen22, 2)}
        if args.ooc_sample > 0:
            c2["out_of_core"] = out_of_core_section(gem, args, local, g22)
        del g22
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    achieved = (jb / jt / 1e9) if jt > 0 else 0.0
    set_names = ",".join(f"{k}{'s' if d == 1 else 'd' if d == 2 else 'a'}" for k, d in sets)
    traffic, traffic_src = profiled_traffic(f"{args.workload} {set_names} batch {B}")
    line = {
        "metric": METRIC,
        "value": exact / tdev if tdev > 0 else 0.0,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": tdev * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32/u64",
        "data": "synthetic R-MAT graph and random-walk queries (seeded)",
        "config": dict(desc, batch=B, query_sets=[f"{k}{'s' if d == 1 else 'd' if d == 2 else 'a'}" for k, d in sets],
                       time_cap_ms=args.cap_ms, parallelism=f"replicas{world}", l2="flushed (256 MiB write)",
                       exact_queries=exact, capped_queries=capped, graph_gen_s=round(gen_s, 2)),
        "embeddings_per_s": emb / tdev if tdev > 0 else 0.0,
        "batched_over_plain": (exact / tdev) / plain["queries_per_s"] if plain.get("queries_per_s") else None,
        "plain": plain,
        "phase_ms": {k: round(v, 3) for k, v in phase.items()},
        "autotune": tuned,
        "serving": serving,
        "rmat22": c2,
        "e2e": {"value": e2e_exact / twall if twall > 0 else 0.0, "unit": "queries/s", "counts_equal": e2e_same,
                "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic, "traffic_source": traffic_src,
                     "alg_bytes_per_launch": jb / n_joins if n_joins else None, "kernel": "join_kernel<COUNT>",
                     "peak_source": peak_src},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if args.cpu_sample > 0:
        line["cpu_baseline"] = cpu_baseline(g, pool, args)
        line["host_path"] = host_path_baseline(g, pool[:B], (phase["filter"] + phase["tables"]) / args.steps)
    print(json.dumps(line), flush=True)


def serving_section(gem, args, local, g, pool, ref_counts):
    """Continuous batching through gem_submit / gem_poll under Poisson arrivals
    of the headline queries (cycled), one stream per rate: latency from the
    arrival to the result being visible, achieved rate, and every count
    checked against the batched run's."""
    import collections
    import random
    out = {"queries": "the headline pool, cycled", "seconds_per_rate": args.serve_seconds, "rates": []}
    with gem.Context(device=local, time_cap_ms=args.cap_ms) as c:
        c.load_graph(g)
        for lam in [float(x) for x in args.serve_rates.split(",") if x]:
            rng = random.Random(0x5E12 + int(lam))
            arr, t = [], 0.0
            while True:
                t += rng.expovariate(lam)
                if t > args.serve_seconds:
                    break
                arr.append(t)
            pending, lat, same, busy, i = collections.deque(), [], True, 0, 0
            t0 = time.perf_counter()
            while i < len(arr) or pending:
                now = time.perf_counter() - t0
                while i < len(arr) and arr[i] <= now:
                    qi = i % len(pool)
                    tk = c.submit(pool[qi])
                    if tk is None:  # admission busy: the arrival waits
                        busy += 1
                        break
                    pending.append((tk, arr[i], qi))
                    i += 1
                while pending:  # oldest first
                    tk, ta, qi = pending[0]
                    r = c.poll(tk)
                    if r is None:
                        break
                    lat.append((time.perf_counter() - t0 - ta) * 1e3)
                    same &= r["status"] == "OK" and r["count"] == ref_counts[qi]
                    pending.popleft()
                if not pending and i < len(arr):
                    time.sleep(max(0.0, arr[i] - (time.perf_counter() - t0)))
            wall = time.perf_counter() - t0
            out["rates"].append({"lambda_qps": lam, "queries": len(lat), "achieved_qps": len(lat) / wall,
                                 "p50_ms": pctl(lat, 50), "p99_ms": pctl(lat, 99), "counts_equal_batched": same,
                                 "admission_busy": busy})
    return out


def profiled_traffic(key):
    """DRAM bytes (read + write) of one join launch of the workload `key`
    ("<workload> <query sets> batch <B>"), from the committed ncu capture
    summary whose `workload_key` line equals it, or None."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "join_*.md"))):
        text = open(path).read()
        k = re.search(r"^workload_key: (.+)$", text, re.M)
        m = re.search(r"^dram_bytes_per_launch: (\d+)$", text, re.M)
        if k and m and k.group(1).strip() == key:
            return int(m.group(1)), os.path.relpath(path, ROOT) + " (ncu, one launch)"
    return None, None


def rmat22_section(gem, args, local, g, gen_s):
    """Scale-22 R-MAT with 16 Zipf(1.0) labels and the 8s/8d/16s/16d query sets:
    per query, plain run under a device time cap (status, count, nodes/s)."""
    per = max(1, args.c2_sample // len(SETS))
    out = {"workload": "rmat22-ef16-zipf16", "time_cap_ms": args.c2_cap_ms, "graph_gen_s": round(gen_s, 2),
           "queries": []}
    with gem.Context(device=local, time_cap_ms=args.c2_cap_ms) as c:
        c.load_graph(g)
        for i, (k, d) in enumerate(SETS):
            for q in gem.gen_queries(g, k, d, per, seed=0x51000 + i):
                r = c.run(q, raise_on_error=False)
                js = r["ms"]["join"] / 1e3
                out["queries"].append({"set": f"{k}{'s' if d == 1 else 'd'}", "edges": q.ne, "status": r["status"],
                                       "count": r["count"] if r["status"] == "OK" else None,
                                       "count_before_cap": r["count"] if r["status"] != "OK" else None,
                                       "join_ms": round(r["ms"]["join"], 1),
                                       "prefix_matches_per_s": r["nodes"] / js if js > 0 else None})
    out["exact"] = sum(1 for x in out["queries"] if x["status"] == "OK")
    return out


def out_of_core_section(gem, args, local, g):
    """The scale-22 graph out of core: one batch of random-walk 4-vertex queries
    run in core, out of core with streamed adjacency partitions and out of
    core reading the pinned adjacency in place.  Per mode the median over 3
    batches of the table-build and wave device times (CUDA events) and the
    streaming counters; the counts must be equal in every mode."""
    import torch
    dev = torch.device("cuda", local)
    h = torch.empty((64 << 20) // 4, dtype=torch.int32).pin_memory()
    d = torch.empty(h.shape, dtype=torch.int32, device=dev)
    for _ in range(3):
        d.copy_(h, non_blocking=True)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(8):
        d.copy_(h, non_blocking=True)
    e1.record()
    torch.cuda.synchronize(dev)
    h2d_gbs = 8 * (64 << 20) / (e0.elapsed_time(e1) * 1e-3) / 1e9
    del h, d
    qs = gem.gen_queries(g, 4, gem.ANY, args.ooc_sample, seed=0x00C0)
    out = {"queries": len(qs), "query_set": "4a", "adjacency_bytes": 4 * int(g.info()["n_arcs"]),
           "pinned_h2d_gbs": round(h2d_gbs, 1), "modes": {}}
    counts = {}
    for name, kw in (("in_core", {}), ("streamed", dict(ooc=True, ooc_stream=1)),
                     ("in_place", dict(ooc=True, ooc_stream=2))):
        with gem.Context(device=local, time_cap_ms=args.c2_cap_ms * 10, **kw) as c:
            c.load_graph(g)
            c.batch(qs)
            tab, tot = [], []
            for _ in range(3):
                _, rs = c.batch(qs)
                waves = {}
                for r in rs:
                    waves.setdefault(r["wave"], r)
                tab.append(sum(w["ms"]["tables"] for w in waves.values()))
                tot.append(sum(w["ms"]["total"] for w in waves.values()))
            counts[name] = [r["count"] if r["status"] == "OK" else None for r in rs]
            m = {"tables_ms": round(sorted(tab)[1], 2), "wave_ms": round(sorted(tot)[1], 2)}
            if kw:
                m["stats"] = c.ooc_stats()
            out["modes"][name] = m
    out["counts_equal"] = all(v == counts["in_core"] for v in counts.values()) and None not in counts["in_core"]
    return out


def host_path_baseline(g, qs, gpu_ms_per_step):
    """The reference's host-side path for one batch: its out-of-core filter and
    edge-table build (OpenMP, out-of-core/lib/filter/src/filter.cu:61-295 and
    out-of-core/lib/structure/src/unifiedTrie.cu:1224-1427, restated in the
    oracle with the reference's worker counts) on the host cores, beside the
    GPU's filter + tables phases per step.  The reference builds both
    directions of every query edge whose source has query degree > 1."""
    import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ntab = 0
    for q in qs:
        cand = oracle.filter_mt(g, q)
        deg = np.bincount(q.edges.reshape(-1), minlength=q.nv) if q.ne else np.zeros(q.nv, int)
        for a, b in q.edges.tolist():
            for s, t in ((a, b), (b, a)):
                if deg[s] > 1:
                    oracle.edge_table_mt(g, cand[s], cand[t])
                    ntab += 1
    ms = (time.perf_counter() - t0) * 1e3
    return {"filter_tables_ms_per_batch": round(ms, 2), "gpu_filter_tables_ms_per_step": round(gpu_ms_per_step, 3),
            "gpu_speedup": round(ms / gpu_ms_per_step, 1) if gpu_ms_per_step > 0 else None,
            "threads": {"filter": min(16, cores), "tables": min(4, cores)}, "queries": len(qs), "tables": ntab,
            "kind": "port"}


def cpu_baseline(g, pool, args):
    import oracle
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    n_ok = 0
    n = 0
    for q in pool[: args.cpu_sample]:
        c, h, ok = oracle.count(g, q, threads=threads, want_hash=False, work_cap=args.cpu_work_cap)
        n += 1
        n_ok += 1 if ok else 0
    dt = time.perf_counter() - t0
    return {"value": n_ok / dt if dt > 0 else 0.0, "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"first {n} queries of the pool, each capped at {args.cpu_work_cap} scanned arcs; "
                      f"{n_ok} completed in {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import gem_b200 as gem
    g, desc, sets, _ = make_workload(gem, args.workload, args.sets)
    pool = query_pool(gem, g, sets, args.per_set)
    import oracle
    threads = os.cpu_count() or 1
    B = args.batch
    S = max(1, min(args.ref_sample, B))
    times, exact, emb = [], 0, 0
    for s in range(args.warmup + args.steps):
        # a bounded sample of the workload per step: S queries, cycling through the pool
        qs = [pool[(s * S + j) % len(pool)] for j in range(S)]
        t0 = time.perf_counter()
        for q in qs:
            c, h, ok = oracle.count(g, q, threads=threads, want_hash=False, work_cap=args.cpu_work_cap)
            if s >= args.warmup and ok:
                exact += 1
                emb += c
        if s >= args.warmup:
            times.append(time.perf_counter() - t0)
    T = sum(times)
    v = exact / T if T > 0 else 0.0
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": T * 1e3 / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64", "data": "synthetic (seeded)",
        "config": dict(desc, batch=B, cpu_work_cap=args.cpu_work_cap),
        "embeddings_per_s": emb / T if T > 0 else 0.0,
        "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"{S} queries per step, cycling through the {len(pool)}-query pool, each capped at "
                                   f"{args.cpu_work_cap} scanned arcs"},
        "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gem", choices=["gem", "reference"])
    ap.add_argument("--workload", default="rmat16")
    ap.add_argument("--sets", default=None, help="query sets, e.g. '8s,8d,16s,16d' (s sparse, d dense, a any)")
    ap.add_argument("--per-set", type=int, default=100)
    ap.add_argument("--batch", type=int, default=100)
    ap.add_argument("--cap-ms", type=int, default=20000)
    ap.add_argument("--plain", type=int, default=100)
    ap.add_argument("--autotune", type=int, default=1)
    ap.add_argument("--c2-sample", type=int, default=8, help="scale-22 queries in the rmat22 section (0 = skip)")
    ap.add_argument("--ooc-sample", type=int, default=50,
                    help="4-vertex queries of the out-of-core comparison on the scale-22 graph (0 = skip)")
    ap.add_argument("--c2-cap-ms", type=int, default=1000)
    ap.add_argument("--cpu-sample", type=int, default=100, help="pool queries timed on the CPU oracle (0 = skip)")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="per arrival rate in the serving section (0 = skip)")
    ap.add_argument("--serve-rates", default="1000,5000,20000", help="Poisson arrival rates (queries/s)")
    ap.add_argument("--cpu-work-cap", type=int, default=1_000_000_000)
    ap.add_argument("--ref-sample", type=int, default=8, help="queries per step of the reference arm (--impl reference)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gem(args)


if __name__ == "__main__":
    main()
