"""Runs the reference's own in-core binary on small seeded inputs and records
the counts it prints, as a fixture that pins the oracle to the reference.

The binary is built from the reference's sources by oracle/ref/Makefile into
oracle/_ref/GEM_ic and needs a GPU.  Inputs stay inside the reference's
envelope: at most 16 query vertices and 16 query edges (in-core
lib/utils/include/defs.h:20-21), at least 2 query edges (its `relax` returns no
relaxed query for one edge, in-core/lib/plan/src/relax.cpp:89-90), and
threshold 0 passed explicitly (its default is 2).  The reference prints the
count through a uint32_t (in-core/src/main.cu:233), so the fixture stores the
printed value, which equals the true count mod 2^32.

Each run of the binary spends most of its time starting up (about half a
minute), so the case list is short and skips queries whose counts run into
the billions; the fixture is rewritten after every case and the run stops
starting new cases once `budget_s` seconds have passed.

With a threshold argument > 0 the binary runs relaxed matching (-t T) on a
smaller list of queries (at most RELAXED_MAX_EDGES edges) and prints one
count per relaxed query; all of them are recorded with their edge sets.

Usage (on a GPU machine):
    python tests/golden/make_ref_counts.py <out.json> [work_dir] [budget_s] [threshold]
"""
import json
import os
import re
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import gem_b200 as gem  # noqa: E402

GRAPHS = [
    # name, scale, edge factor, labels, zipf s, seed, [(query vertices, density), ...]
    ("rmat10_l3", 10, 8, 3, 0.0, 0x5201, [(3, gem.ANY), (4, gem.ANY), (4, gem.SPARSE), (5, gem.ANY), (6, gem.DENSE)]),
    ("rmat11_l6z", 11, 8, 6, 1.0, 0x5202, [(4, gem.ANY), (5, gem.SPARSE), (6, gem.SPARSE)]),
    ("rmat12_l8", 12, 8, 8, 0.0, 0x5203, [(4, gem.SPARSE), (6, gem.SPARSE)]),
]
# The binary ended with CUDA error 700 (illegal address; exit code 188 through
# in-core/lib/utils/include/cuda_helpers.cuh:34) on two queries of 11 and 12
# edges (7 vertices dense on rmat11_l6z, 8 vertices sparse on rmat12_l8).
# Those sizes are left out and no query with more than MAX_QUERY_EDGES edges
# is run.
MAX_QUERY_EDGES = 10
GRAPHS_RELAXED = [
    ("rmat10_l3", 10, 8, 3, 0.0, 0x5201, [(4, gem.ANY), (4, gem.DENSE), (5, gem.ANY), (5, gem.DENSE)]),
    ("rmat11_l6z", 11, 8, 6, 1.0, 0x5202, [(4, gem.ANY), (5, gem.DENSE)]),
]
RELAXED_MAX_EDGES = 8
PER_SIZE = 2


def main():
    out = sys.argv[1]
    work = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(out), "ref_inputs")
    budget_s = float(sys.argv[3]) if len(sys.argv) > 3 else 1e9
    threshold = int(sys.argv[4]) if len(sys.argv) > 4 else 0
    graphs = GRAPHS_RELAXED if threshold else GRAPHS
    max_edges = RELAXED_MAX_EDGES if threshold else MAX_QUERY_EDGES
    binary = os.path.join(ROOT, "oracle", "_ref", "GEM_ic")
    os.makedirs(work, exist_ok=True)
    cases = []
    t_start = time.time()

    def save():
        with open(out, "w") as f:
            json.dump({"binary": "oracle/_ref/GEM_ic (in-core, built by oracle/ref/Makefile)", "threshold": threshold,
                       "cases": cases}, f, indent=0)

    for gname, scale, ef, nl, zs, seed, sizes in graphs:
        g = gem.HostGraph.rmat(scale, ef, seed=seed).set_labels(nl, zs, seed=seed ^ 0x4C)
        gpath = os.path.join(work, gname + ".graph")
        g.write_text(gpath)
        gd = dict(name=gname, scale=scale, edge_factor=ef, labels=nl, zipf_s=zs, seed=seed)
        for (k, dens) in sizes:
            for i, q in enumerate(gem.gen_queries(g, k, dens, PER_SIZE, seed=seed * 131 + k * 7 + dens)):
                if q.ne < 2 or q.ne > max_edges or q.nv > 16:
                    continue
                if time.time() - t_start > budget_s:
                    print("budget reached", flush=True)
                    return
                qpath = os.path.join(work, f"{gname}_k{k}_d{dens}_{i}.in")
                q.write_text(qpath)
                t0 = time.time()
                try:
                    r = subprocess.run([binary, "-q", qpath, "-d", gpath, "-t", str(threshold), "-g", "0"],
                                       capture_output=True,
                                       text=True, timeout=120)
                    m = re.findall(r"Relaxed Query ET ([01]+): (\d+) matches", r.stdout)
                    rec = dict(graph=gd, labels=q.labels.tolist(), edges=q.edges.tolist(), exit=r.returncode,
                               printed=[int(c) for _, c in m], et=[e for e, _ in m])
                except subprocess.TimeoutExpired:
                    rec = dict(graph=gd, labels=q.labels.tolist(), edges=q.edges.tolist(), exit="timeout", printed=[],
                               et=[])
                rec["elapsed_s"] = round(time.time() - t0, 2)
                cases.append(rec)
                save()
                print(gname, k, dens, i, rec["exit"], rec["printed"], rec["elapsed_s"], flush=True)


if __name__ == "__main__":
    main()
