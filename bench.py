#!/usr/bin/env python3
"""Benchmark: exact subgraph-matching throughput on one B200 (queries/s and
embeddings/s, batched vs plain, p50/p99 latency).

Headline workload (`--workload rmat22-mix`, the batched configuration):
R-MAT scale 22 (4,194,304 vertices), edge factor 16, (a,b,c,d) =
(0.57,0.19,0.19,0.05), self loops and duplicates removed, uint32 CSR with
sorted adjacency, 16 labels Zipf(s=1.0); 1,000 random-walk queries whose
sizes are drawn uniformly from {4, 8, 12, 16, 24, 32} vertices, alternately
sparse (average degree <= 3) and dense (above 3; a 4-vertex query cannot
exceed 3, so its "dense" draw keeps the walk's induced edges).  Seeded
synthetic stand-ins; the reference's datasets are not used.  A step is one
gem_batch_run over the 1,000 queries.  Every query runs under a per-query
device time cap (`--cap-ms`): a query still running when the cap expires is
reported as capped, never as an exact count, and the headline counts exact
queries only.  `plain` runs a stratified sample of the same queries one
gem_query_run each under the same cap.

Section `config1` (`--workload rmat16` makes it the headline): R-MAT scale
16, edge factor 8, 8 uniform labels, 100 random-walk 4-vertex queries, all
exact; batched vs plain, every count and hash checked against the CPU oracle.
Its `serving` part submits those queries through gem_submit / gem_poll under
Poisson arrivals.

Section `rmat22`: the scale-22 graph with the 8s/8d/16s/16d query sets, each
query plain under a device cap (status and prefix-match rate).  Its
`out_of_core` part runs 4-vertex queries in core, out of core with streamed
adjacency partitions and out of core reading the pinned adjacency in place.

`value` is device-timed (CUDA events, from each step's first kernel to its
last, inputs resident in HBM), `e2e` is wall time around the same C-ABI
calls from host buffers
(query arrays in, results out).  L2 is flushed between steps (a 256 MiB
write).  With torchrun (N > 1) every rank runs an independent replica on its
own queries (the path has no exchange step); rank 0 reports the max time.
`--impl reference` times the CPU restatement of the path (the reference has
no CPU join) on the host cores with all threads; it builds its inputs with
the oracle's generators and never loads libgem.
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
MIX_SIZES = (4, 8, 12, 16, 24, 32)
METRIC = "queries/s & embeddings/s on 1 B200, batched vs plain, exact counts; p50/p99 ms"
GRAPHS = {  # name: (scale, edge factor, labels, zipf s)
    "rmat22-mix": (22, 16, 16, 1.0),
    "rmat16": (16, 8, 8, 0.0),
    "rmat22": (22, 16, 16, 1.0),
}
DEFAULTS = {  # per workload: batch, per-query cap (ms), plain sample, autotune
    "rmat22-mix": dict(batch=1000, cap_ms=100, plain=200, autotune=0),
    "rmat16": dict(batch=100, cap_ms=20000, plain=100, autotune=1),
}


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


def _mix64(x):
    """splitmix64 finaliser of x + golden gamma (the generators' mixer)."""
    m = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & m
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    return x ^ (x >> 31)


def make_graph(backend, name):
    """The seeded data graph of a workload, built by `backend`: the libgem
    binding (gem_b200) or the oracle's restated generators (same arrays)."""
    scale, ef, nl, zs = GRAPHS[name]
    seed = 0x47454D00 + scale
    t = time.time()
    if backend.__name__ == "oracle":
        g = backend.set_labels(backend.rmat(scale, ef, seed=seed), nl, zs, seed=seed ^ 0x4C)
    else:
        g = backend.HostGraph.rmat(scale, ef, seed=seed).set_labels(nl, zs, seed=seed ^ 0x4C)
    return g, time.time() - t


def mix_pool(backend, g, n, seed=0x51003, sizes=MIX_SIZES):
    """Config-3 queries: query i has size MIX_SIZES[mix64(seed + i) % 6] and is
    sparse for even i, dense for odd i; the queries of one (size, density)
    come from one random-walk stream (seed << 8 | 4 size + density)."""
    ks = [sizes[_mix64(seed + i) % len(sizes)] for i in range(n)]
    ds = [1 + (i % 2) for i in range(n)]
    need = {}
    for k, d in zip(ks, ds):
        need[(k, d)] = need.get((k, d), 0) + 1
    made = {kd: backend.gen_queries(g, kd[0], kd[1], c, seed=(seed << 8) | (4 * kd[0] + kd[1]))
            for kd, c in need.items()}
    used = {kd: 0 for kd in need}
    out = []
    for k, d in zip(ks, ds):
        out.append(made[(k, d)][used[(k, d)]])
        used[(k, d)] += 1
    return out


def config1_pool(backend, g, n=100, seed=0x51000):
    return backend.gen_queries(g, 4, 0, n, seed=seed)


def workload_pool(backend, name, g, n, sizes=MIX_SIZES):
    if name == "rmat22-mix":
        return mix_pool(backend, g, n, sizes=sizes)
    if name == "rmat16":
        return config1_pool(backend, g, n)
    raise SystemExit(f"unknown workload {name}")


def workload_config(name, args, world):
    """The `config` object both arms print for a workload."""
    scale, ef, nl, zs = GRAPHS[name]
    c = {"workload": f"{name}-ef{ef}-{'zipf' if zs else 'uniform'}{nl}" if name != "rmat22-mix"
         else "rmat22-ef16-zipf16-mix1000", "scale": scale, "edge_factor": ef, "labels": nl, "zipf_s": zs,
         "batch": args.batch, "time_cap_ms": args.cap_ms, "parallelism": f"replicas{world}",
         "l2": "flushed (256 MiB write)"}
    if name == "rmat22-mix":
        c["query_sizes"] = list(args.sizes)
        c["densities"] = "alternating sparse/dense"
    else:
        c["query_sizes"] = [4]
    return c


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


def waves_of(rs):
    w = {}
    for r in rs:
        w.setdefault(r["wave"], r)
    return list(w.values())


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
    g, gen_s = make_graph(gem, args.workload)
    B = args.batch
    pool = workload_pool(gem, args.workload, g, B * world, args.sizes)
    ctx = gem.Context(device=local, time_cap_ms=args.cap_ms, batch_lanes=args.lanes)
    ctx.load_graph(g)
    tuned = {}
    if args.autotune:
        # tuned on a disjoint sample of the same configuration (another query seed)
        tune_pool = config1_pool(gem, g, B, seed=0x51080) if args.workload == "rmat16" else mix_pool(gem, g, B, 0x51083)
        tuned = ctx.autotune(tune_pool, trial_cap_ms=args.cap_ms)

    def batch_of(step):
        return [pool[i] for i in batch_indices(step, rank, world, B, len(pool))]

    for s in range(args.warmup):
        ctx.batch(batch_of(s))
    steps = list(range(args.warmup, args.warmup + args.steps))
    dev_ms, wall_ms, res_all = [], [], []
    h2d = d2h = launches = 0
    jbytes = jms = tbytes = tpass_ms = busy_ms = 0.0
    n_joins = n_tab = 0
    phase = {"filter": 0.0, "tables": 0.0, "index": 0.0, "join": 0.0}
    with Clocks(local) as clk:
        for s in steps:
            qs = batch_of(s)
            flush_l2(dev)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st, rs = ctx.batch(qs)  # query arrays from host memory, results back in host memory
            torch.cuda.synchronize()
            wall_ms.append((time.perf_counter() - t0) * 1e3)
            ws = waves_of(rs)
            # device time of the step: its first wave's first event to its last
            # wave's last event (CUDA events on one timeline), so a wave retried
            # after an out-of-memory split and the gaps between waves count too
            dev_ms.append(max(r["t_end_ms"] for r in ws) - min(r["t_begin_ms"] for r in ws))
            busy_ms += sum(r["ms"]["total"] for r in ws)
            launches += sum(r["launches"] for r in ws)
            jbytes += sum(r["bytes_alg"][3] for r in ws)
            jms += sum(r["ms"]["join"] for r in ws)
            n_joins += len(ws)
            for r in ws:
                if r["table_pass_ms"][0] + r["table_pass_ms"][1] > 0:
                    tbytes += r["bytes_alg"][2]
                    tpass_ms += r["table_pass_ms"][0] + r["table_pass_ms"][1]
                    n_tab += 1
            for k in phase:
                phase[k] += sum(r["ms"][k] for r in ws)
            h2d += sum(4 * q.nv + 8 * q.ne for q in qs)  # the queries' label and edge arrays
            d2h += ctypes_result_bytes(gem) * len(qs)
            res_all.append(rs)
    exact = sum(1 for rs in res_all for r in rs if r["status"] == "OK")
    capped = sum(1 for rs in res_all for r in rs if r["status"] == "ERR_TIMEOUT")
    emb = sum(r["count"] for rs in res_all for r in rs if r["status"] == "OK")
    counts_stable = all(res_all[0][i]["count"] == rs[i]["count"] for rs in res_all[1:] for i in range(len(rs))
                        if rs[i]["status"] == "OK" and res_all[0][i]["status"] == "OK") if world == 1 else None
    tdev = sum(dev_ms) / 1e3
    twall = sum(wall_ms) / 1e3
    e2e_exact = exact
    if dist:
        tdev, twall, exact, emb, capped, e2e_exact = reduce_over_ranks(dist, tdev, twall, exact, emb, capped, exact)
    plain = {}
    if rank == 0 and args.plain > 0:
        plain = plain_section(ctx, batch_of(args.warmup), res_all[0], args.plain)
    ctx.close()
    sections = {}
    if rank == 0 and args.workload == "rmat22-mix" and args.serve5_seconds > 0:
        ref5 = {i: r["count"] for i, r in enumerate(res_all[0]) if r["status"] == "OK"}
        sections["serving"] = serving_section(gem, local, g, batch_of(args.warmup), ref5,
                                              [float(x) for x in args.serve5_rates.split(",") if x],
                                              args.serve5_seconds, args.cap_ms, 120,
                                              label="the scale-22 mixed-size pool")
    if rank == 0 and args.workload != "rmat16" and args.config1:
        sections["config1"] = config1_section(gem, args, local)
    if rank == 0 and (args.c2_sample > 0 or args.ooc_sample > 0):
        if args.workload.startswith("rmat22"):
            g22, gen22 = g, gen_s
        else:
            g22, gen22 = make_graph(gem, "rmat22")
        c2 = rmat22_section(gem, args, local, g22, gen22) if args.c2_sample > 0 else {"graph_gen_s": round(gen22, 2)}
        if args.ooc_sample > 0:
            c2["out_of_core"] = out_of_core_section(gem, args, local, g22)
        sections["rmat22"] = c2
        del g22
    if rank == 0 and args.ooc26:
        sections["out_of_core_scale26"] = ooc26_section(gem, args, local)
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    cfg = workload_config(args.workload, args, world)
    value = exact / tdev if tdev > 0 else 0.0
    line = {
        "metric": METRIC,
        "value": value,
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
        "config": cfg,
        "exact_queries": exact,
        "capped_queries": capped,
        "graph_gen_s": round(gen_s, 2),
        "embeddings_per_s": emb / tdev if tdev > 0 else 0.0,
        "embeddings_note": "sum of the exact queries' counts per second; closed-form suffix levels are counted, "
                           "not enumerated one by one",
        "batched_over_plain": value / plain["queries_per_s"] if plain.get("queries_per_s") else None,
        "plain": plain,
        "counts_stable_across_steps": counts_stable,
        "phase_ms_per_step": {k: round(v / args.steps, 3) for k, v in phase.items()},
        "waves_busy_ms_per_step": round(busy_ms / args.steps, 3),
        "autotune": tuned,
        "e2e": {"value": e2e_exact / twall if twall > 0 else 0.0, "unit": "queries/s",
                "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    # roofline of the dominant kernel: the edge-table passes or the join
    t_tab = tpass_ms / n_tab if n_tab else 0.0
    t_join = jms / n_joins if n_joins else 0.0
    roof_tab = roofline(tbytes / n_tab if n_tab else 0.0, t_tab, peak, peak_src,
                        "table_vtx_kernel<count>+<write> (edge-table passes over vertex tiles)",
                        profiled_traffic("tables", args.workload, B))
    roof_join = roofline(jbytes / n_joins if n_joins else 0.0, t_join, peak, peak_src, "join_kernel<COUNT>",
                         profiled_traffic("join", args.workload, B))
    line["roofline"], line["roofline_other"] = (roof_tab, roof_join) if tpass_ms >= jms else (roof_join, roof_tab)
    line["roofline"]["share_of_step"] = round((tpass_ms if tpass_ms >= jms else jms) / (tdev * 1e3), 3) if tdev else None
    if args.cpu_sample > 0:
        line["parity"] = oracle_parity(g, batch_of(args.warmup), res_all[0], args.cpu_parity_cap, args.parity_budget_s)
        line["cpu_baseline"] = cpu_baseline(g, pool, args)
        qs0 = batch_of(args.warmup)
        hstride = max(1, len(qs0) // args.host_path_queries)
        line["host_path"] = host_path_baseline(g, qs0[::hstride], (phase["filter"] + phase["tables"]) / args.steps,
                                               len(qs0), args.cpu_budget_s)
    line.update(sections)
    print(json.dumps(line), flush=True)


def ctypes_result_bytes(gem):
    import ctypes
    return ctypes.sizeof(gem._Result)


def roofline(alg_bytes, ms, peak, peak_src, kernel, traffic):
    achieved = alg_bytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    ratio, src = traffic
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak if peak else None,
            "traffic": int(ratio * alg_bytes) if ratio is not None else None,
            "traffic_source": src, "alg_bytes_per_launch": alg_bytes, "ms_per_launch": ms,
            "kernel": kernel, "peak_source": peak_src}


def profiled_traffic(kind, workload, batch=None):
    """DRAM bytes (read + write) per algorithmic byte of `kind` ("join" or
    "tables") on `workload`, from the committed ncu capture summary whose
    `workload_key` line is "<kind> <workload>" and which states
    `dram_per_alg_byte` (the ratio does not depend on the wave's size, so a
    capture of a smaller wave scales to the bench's launches), or (None, None)."""
    import glob
    import re
    key = f"{kind} {workload}"
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        text = open(path).read()
        k = re.search(r"^workload_key: (.+)$", text, re.M)
        m = re.search(r"^dram_per_alg_byte: ([0-9.]+)$", text, re.M)
        if k and m and k.group(1).strip() == key:
            return float(m.group(1)), os.path.relpath(path, ROOT) + " (ncu DRAM bytes / algorithmic bytes of a capture)"
    return None, None


def plain_section(ctx, qs_all, batch_res, n):
    """The same queries one gem_query_run each (a stratified sample of n of
    them: every len/n-th), same cap; device time from CUDA events, latency
    on the host; counts compared with the batched run where both are exact."""
    import torch
    stride = max(1, len(qs_all) // n)
    idx = list(range(0, len(qs_all), stride))[:n]
    lat, pe, pn, pdev, same, capped = [], 0, 0, 0.0, True, 0
    bexact = 0
    for i in idx:
        q = qs_all[i]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = ctx.run(q, raise_on_error=False)
        torch.cuda.synchronize()
        lat.append((time.perf_counter() - t0) * 1e3)
        pdev += r["ms"]["total"] / 1e3
        rb = batch_res[i]
        bexact += rb["status"] == "OK"
        if r["status"] == "OK":
            pn += 1
            pe += r["count"]
            same &= rb["status"] != "OK" or rb["count"] == r["count"]
        elif r["status"] == "ERR_TIMEOUT":
            capped += 1
    return {"queries": len(idx), "sample": f"every {stride}th query of the batch", "exact": pn, "capped": capped,
            "batched_exact_same_queries": bexact,
            "queries_per_s": pn / pdev if pdev else None, "queries_per_s_wall": pn / (sum(lat) / 1e3) if lat else None,
            "embeddings_per_s": pe / pdev if pdev else None,
            "p50_ms": pctl(lat, 50), "p99_ms": pctl(lat, 99), "counts_equal_batched": same}


def config1_section(gem, args, local):
    """Configuration 1 (R-MAT scale 16, 100 four-vertex queries): batched vs
    plain, every count checked against the oracle, and serving."""
    import torch
    dev = torch.device("cuda", local)
    g, gen_s = make_graph(gem, "rmat16")
    pool = config1_pool(gem, g)
    out = {"workload": "rmat16-ef8-uniform8", "queries": len(pool), "graph_gen_s": round(gen_s, 2)}
    with gem.Context(device=local, time_cap_ms=20000) as c:
        c.load_graph(g)
        out["autotune"] = c.autotune(config1_pool(gem, g, 100, seed=0x51080), trial_cap_ms=20000)
        for _ in range(3):
            c.batch(pool)
        ts, rs = [], None
        for _ in range(args.c1_steps):
            flush_l2(dev)
            _, rs = c.batch(pool)
            ws = waves_of(rs)
            ts.append(max(r["t_end_ms"] for r in ws) - min(r["t_begin_ms"] for r in ws))
        exact = sum(r["status"] == "OK" for r in rs)
        out["batched_queries_per_s"] = exact / (sum(ts) / len(ts) / 1e3)
        out["batched_ms_per_step"] = statistics.median(ts)
        out["plain"] = plain_section(c, pool, rs, len(pool))
        out["batched_over_plain"] = (out["batched_queries_per_s"] / out["plain"]["queries_per_s"]
                                     if out["plain"].get("queries_per_s") else None)
        counts = [r["count"] if r["status"] == "OK" else None for r in rs]
    out["parity"] = oracle_parity(g, pool, rs, 0, 120.0)
    if args.serve_seconds > 0:
        out["serving"] = serving_section(gem, local, g, pool, {i: x for i, x in enumerate(counts)},
                                         [float(x) for x in args.serve_rates.split(",") if x], args.serve_seconds,
                                         20000, label="the config-1 pool")
    return out


def oracle_parity(g, qs, rs, work_cap, budget_s):
    """The batched run's exact counts against the CPU oracle (each query under
    `work_cap` scanned arcs, 0 = none; queries the oracle does not finish
    are skipped and counted; stops starting queries after budget_s)."""
    import oracle
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    checked = equal = skipped = 0
    for q, r in zip(qs, rs):
        if r["status"] != "OK":
            continue
        if time.perf_counter() - t0 > budget_s:
            skipped += 1
            continue
        c, _, ok = oracle.count(g, q, threads=threads, want_hash=False, work_cap=work_cap)
        if not ok:
            skipped += 1
            continue
        checked += 1
        equal += c == r["count"]
    return {"checked": checked, "equal": equal, "not_finished_by_oracle": skipped,
            "oracle_work_cap": work_cap, "seconds": round(time.perf_counter() - t0, 1)}


def serving_section(gem, local, g, pool, ref_counts, rates, seconds, cap_ms, admit_gb=0, label="the pool"):
    """Continuous batching through gem_submit / gem_poll under Poisson arrivals
    of the pool's queries (cycled), one stream per rate: latency from the
    arrival to the result being visible, achieved rate, exact and capped
    results, and every exact count checked against the batched run's."""
    import collections
    import random
    out = {"queries": f"{label}, cycled", "seconds_per_rate": seconds, "time_cap_ms": cap_ms,
           "admission_budget_gib": admit_gb or 120, "rates": []}
    with gem.Context(device=local, time_cap_ms=cap_ms, admit_gb=admit_gb) as c:
        c.load_graph(g)
        for lam in rates:
            rng = random.Random(0x5E12 + int(lam))
            arr, t = [], 0.0
            while True:
                t += rng.expovariate(lam)
                if t > seconds:
                    break
                arr.append(t)
            pending, lat, same, busy, i = collections.deque(), [], True, 0, 0
            exact = capped = checked = 0
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
                    if r["status"] == "OK":
                        exact += 1
                        if ref_counts.get(qi) is not None:
                            checked += 1
                            same &= r["count"] == ref_counts[qi]
                    elif r["status"] == "ERR_TIMEOUT":
                        capped += 1
                    else:
                        same = False
                    pending.popleft()
                if pending or i < len(arr):
                    time.sleep(0.0002 if pending else max(0.0, arr[i] - (time.perf_counter() - t0)))
            wall = time.perf_counter() - t0
            out["rates"].append({"lambda_qps": lam, "queries": len(lat), "achieved_qps": len(lat) / wall,
                                 "exact": exact, "capped": capped, "exact_qps": exact / wall,
                                 "p50_ms": pctl(lat, 50), "p99_ms": pctl(lat, 99),
                                 "counts_checked": checked, "counts_equal_batched": same, "admission_busy": busy})
    return out


def rmat22_section(gem, args, local, g, gen_s):
    """Scale-22 R-MAT with 16 Zipf(1.0) labels and the 8s/8d/16s/16d query sets:
    per query, plain run under a device time cap (status, nodes/s).  A capped
    query reports the partial embeddings it extended before the cap, not a
    count."""
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
                                       "prefix_matches": r["nodes"], "join_ms": round(r["ms"]["join"], 1),
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
                ws = waves_of(rs)
                tab.append(sum(w["ms"]["tables"] for w in ws))
                tot.append(sum(w["ms"]["total"] for w in ws))
            counts[name] = [r["count"] if r["status"] == "OK" else None for r in rs]
            m = {"tables_ms": round(sorted(tab)[1], 2), "wave_ms": round(sorted(tot)[1], 2)}
            if kw:
                m["stats"] = c.ooc_stats()
            out["modes"][name] = m
    out["counts_equal"] = all(v == counts["in_core"] for v in counts.values()) and None not in counts["in_core"]
    return out


def ooc26_section(gem, args, local):
    """Configuration 4: R-MAT scale 26 (67,108,864 vertices), edge factor 16,
    32 labels Zipf(1.2), the adjacency in pinned host memory and a 24 GiB
    device budget.  100 dense 12-vertex random-walk queries in one batch
    under the per-query cap (waves split to fit the budget), and 4-vertex
    queries run out of core and in core (the 8.6 GB adjacency also fits the
    device) with equal counts."""
    t = time.time()
    g = gem.HostGraph.rmat(26, 16, seed=0x47454D00 + 26).set_labels(32, 1.2, seed=(0x47454D00 + 26) ^ 0x4C)
    out = {"workload": "rmat26-ef16-zipf32(1.2)", "graph_gen_s": round(time.time() - t, 1),
           "adjacency_bytes": 4 * int(g.info()["n_arcs"]), "device_budget_gib": 24, "time_cap_ms": args.ooc26_cap_ms}
    q12 = gem.gen_queries(g, 12, gem.DENSE, 100, seed=0x51400)
    q4 = gem.gen_queries(g, 4, gem.ANY, args.ooc26_small, seed=0x51404)
    with gem.Context(device=local, time_cap_ms=args.ooc26_cap_ms, ooc=True, budget_bytes=24 << 30) as c:
        t = time.time()
        c.load_graph(g)
        out["load_s"] = round(time.time() - t, 1)
        t = time.time()
        _, rs = c.batch(q12)
        ws = waves_of(rs)
        out["dense12"] = {"queries": len(q12), "wall_s": round(time.time() - t, 2), "waves": len(ws),
                          "exact": sum(r["status"] == "OK" for r in rs),
                          "capped": sum(r["status"] == "ERR_TIMEOUT" for r in rs),
                          "other": sorted({r["status"] for r in rs} - {"OK", "ERR_TIMEOUT"}),
                          "phase_ms": {k: round(sum(w["ms"][k] for w in ws), 1) for k in ("filter", "tables", "join")}}
        _, r4 = c.batch(q4)
        ws4 = waves_of(r4)
        out["small4_out_of_core"] = {"queries": len(q4), "waves": len(ws4),
                                     "wave_ms": round(sum(w["ms"]["total"] for w in ws4), 1),
                                     "exact": sum(r["status"] == "OK" for r in r4)}
        out["ooc_stats"] = c.ooc_stats()
    with gem.Context(device=local, time_cap_ms=args.ooc26_cap_ms) as c:
        c.load_graph(g)
        _, r4i = c.batch(q4)
        out["small4_in_core_wave_ms"] = round(sum(w["ms"]["total"] for w in waves_of(r4i)), 1)
    both = [(a["count"], b["count"]) for a, b in zip(r4, r4i) if a["status"] == "OK" and b["status"] == "OK"]
    out["small4_in_core_exact"] = sum(r["status"] == "OK" for r in r4i)
    out["small4_both_exact"] = len(both)
    out["small4_counts_equal"] = all(a == b for a, b in both)
    return out


def host_path_baseline(g, qs, gpu_ms_per_step, step_queries, budget_s):
    """The reference's host-side path for a sample of the batch: its
    out-of-core filter and edge-table build (OpenMP, out-of-core/lib/filter/
    src/filter.cu:61-295 and out-of-core/lib/structure/src/unifiedTrie.cu
    :1224-1427, restated in the oracle with the reference's worker counts) on
    the host cores, scaled to the step's queries, beside the GPU's filter +
    tables phases per step.  The reference builds both directions of every
    query edge whose source has query degree > 1."""
    import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ntab = done = 0
    for q in qs:
        if time.perf_counter() - t0 > budget_s:
            break
        done += 1
        cand = oracle.filter_mt(g, q)
        deg = np.bincount(q.edges.reshape(-1), minlength=q.nv) if q.ne else np.zeros(q.nv, int)
        for a, b in q.edges.tolist():
            for s, t in ((a, b), (b, a)):
                if deg[s] > 1:
                    oracle.edge_table_mt(g, cand[s], cand[t])
                    ntab += 1
    ms = (time.perf_counter() - t0) * 1e3
    per_step = ms * step_queries / max(1, done)
    return {"filter_tables_ms_sample": round(ms, 2), "sample_queries": done,
            "filter_tables_ms_per_step_est": round(per_step, 1),
            "gpu_filter_tables_ms_per_step": round(gpu_ms_per_step, 3),
            "gpu_speedup": round(per_step / gpu_ms_per_step, 1) if gpu_ms_per_step > 0 else None,
            "threads": {"filter": min(16, cores), "tables": min(4, cores)}, "tables": ntab, "kind": "port"}


def cpu_baseline(g, pool, args):
    """The oracle on the host cores over a bounded sample of the pool."""
    import oracle
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    n_ok = n = 0
    stride = 7 if len(pool) % 7 else 1  # spread the sample over the pool's sizes
    for i in range(min(args.cpu_sample, len(pool))):
        q = pool[(i * stride) % len(pool)]
        if time.perf_counter() - t0 > args.cpu_budget_s:
            break
        c, h, ok = oracle.count(g, q, threads=threads, want_hash=False, work_cap=args.cpu_work_cap)
        n += 1
        n_ok += 1 if ok else 0
    dt = time.perf_counter() - t0
    return {"value": n_ok / dt if dt > 0 else 0.0, "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"{n} queries of the pool (every {stride}th), each capped at {args.cpu_work_cap} scanned arcs; "
                      f"{n_ok} completed in {dt:.1f} s"}


def run_reference(args):
    """The reference arm: the CPU restatement of the path (the reference has
    no CPU join) over a bounded sample per step, inputs from the oracle's
    generators (libgem is never loaded)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    g, _ = make_graph(oracle, args.workload)
    pool = workload_pool(oracle, args.workload, g, args.batch, args.sizes)
    threads = os.cpu_count() or 1
    S = max(1, min(args.ref_sample, len(pool)))
    times, exact, emb = [], 0, 0
    stride = 7 if len(pool) % 7 else 1  # spread the sampled queries over the pool's sizes
    for s in range(args.warmup + args.steps):
        qs = [pool[((s * S + j) * stride) % len(pool)] for j in range(S)]
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
    cfg = workload_config(args.workload, args, world)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": T * 1e3 / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64", "data": "synthetic (seeded)", "config": cfg,
        "embeddings_per_s": emb / T if T > 0 else 0.0,
        "cpu_baseline": {"value": v, "unit": "queries/s", "cores": threads, "kind": "port",
                         "sample": f"{S} queries per step, every {stride}th of the {len(pool)}-query pool in turn, "
                                   f"each capped at {args.cpu_work_cap} scanned arcs (a capped query is not counted "
                                   f"as exact)"},
        "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gem", choices=["gem", "reference"])
    ap.add_argument("--workload", default="rmat22-mix", choices=sorted(DEFAULTS))
    ap.add_argument("--batch", type=int, default=None, help="queries per step (default: the workload's)")
    ap.add_argument("--sizes", default=None,
                    help="query sizes of the scale-22 mix, e.g. '4' (default: 4,8,12,16,24,32)")
    ap.add_argument("--cap-ms", type=int, default=None, help="per-query device time cap")
    ap.add_argument("--plain", type=int, default=None, help="queries of the plain sample (0 = skip)")
    ap.add_argument("--autotune", type=int, default=None)
    ap.add_argument("--config1", type=int, default=1, help="run the config-1 section (headline rmat22-mix)")
    ap.add_argument("--lanes", type=int, default=0, help="batch lanes: 0 = two for multi-wave batches, 1 = one")
    ap.add_argument("--c1-steps", type=int, default=10)
    ap.add_argument("--c2-sample", type=int, default=8, help="scale-22 queries in the rmat22 section (0 = skip)")
    ap.add_argument("--ooc-sample", type=int, default=50,
                    help="4-vertex queries of the out-of-core comparison on the scale-22 graph (0 = skip)")
    ap.add_argument("--c2-cap-ms", type=int, default=1000)
    ap.add_argument("--cpu-sample", type=int, default=100, help="pool queries timed on the CPU oracle (0 = skip)")
    ap.add_argument("--cpu-budget-s", type=float, default=20.0, help="wall-time bound of the CPU legs")
    ap.add_argument("--parity-budget-s", type=float, default=60.0, help="wall-time bound of the oracle parity check")
    ap.add_argument("--cpu-parity-cap", type=int, default=2_000_000_000, help="oracle work cap of the parity check")
    ap.add_argument("--host-path-queries", type=int, default=100)
    ap.add_argument("--serve-seconds", type=float, default=1.0,
                    help="per arrival rate in the config-1 serving section (0 = skip)")
    ap.add_argument("--serve-rates", default="1000,5000,20000", help="Poisson arrival rates (queries/s), config 1")
    ap.add_argument("--serve5-seconds", type=float, default=3.0,
                    help="per arrival rate in the scale-22 serving section (0 = skip)")
    ap.add_argument("--serve5-rates", default="50,200,1000", help="Poisson arrival rates (queries/s), scale 22")
    ap.add_argument("--ooc26", type=int, default=0, help="run the scale-26 out-of-core section (minutes)")
    ap.add_argument("--ooc26-cap-ms", type=int, default=1000)
    ap.add_argument("--ooc26-small", type=int, default=20, help="4-vertex queries compared in and out of core")
    ap.add_argument("--cpu-work-cap", type=int, default=1_000_000_000,
                    help="scanned-arc cap per query of the CPU legs and the reference arm")
    ap.add_argument("--ref-sample", type=int, default=2, help="queries per step of the reference arm (--impl reference)")
    args = ap.parse_args(argv)
    args.sizes = tuple(int(x) for x in args.sizes.split(",")) if args.sizes else MIX_SIZES
    d = DEFAULTS[args.workload]
    for k in ("batch", "cap_ms", "plain", "autotune"):
        if getattr(args, k) is None:
            setattr(args, k, d[k])
    return args


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gem(args)


if __name__ == "__main__":
    main()
