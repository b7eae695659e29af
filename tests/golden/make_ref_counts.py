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

Usage (on a GPU machine):
    python tests/golden/make_ref_counts.py <out.json> [work_dir]
"""
import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import gem_b200 as gem  # noqa: E402

GRAPHS = [
    # name, scale, edge factor, labels, zipf s, seed
    ("rmat10_l3", 10, 8, 3, 0.0, 0x5201),
    ("rmat11_l4z", 11, 8, 4, 1.0, 0x5202),
    ("rmat12_l8", 12, 8, 8, 0.0, 0x5203),
]
QUERY_SIZES = [(3, gem.ANY), (4, gem.ANY), (4, gem.SPARSE), (5, gem.ANY), (6, gem.SPARSE), (6, gem.DENSE),
               (8, gem.SPARSE)]
PER_SIZE = 2


def main():
    out = sys.argv[1]
    work = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(out), "ref_inputs")
    binary = os.path.join(ROOT, "oracle", "_ref", "GEM_ic")
    os.makedirs(work, exist_ok=True)
    cases = []
    for gname, scale, ef, nl, zs, seed in GRAPHS:
        g = gem.HostGraph.rmat(scale, ef, seed=seed).set_labels(nl, zs, seed=seed ^ 0x4C)
        gpath = os.path.join(work, gname + ".graph")
        g.write_text(gpath)
        for (k, dens) in QUERY_SIZES:
            for i, q in enumerate(gem.gen_queries(g, k, dens, PER_SIZE, seed=seed * 131 + k * 7 + dens)):
                if q.ne < 2 or q.ne > 16 or q.nv > 16:
                    continue
                qpath = os.path.join(work, f"{gname}_k{k}_d{dens}_{i}.in")
                q.write_text(qpath)
                try:
                    r = subprocess.run([binary, "-q", qpath, "-d", gpath, "-t", "0", "-g", "0"], capture_output=True,
                                       text=True, timeout=120)
                    m = re.findall(r"Relaxed Query ET ([01]+): (\d+) matches", r.stdout)
                    rec = dict(graph=dict(name=gname, scale=scale, edge_factor=ef, labels=nl, zipf_s=zs, seed=seed),
                               labels=q.labels.tolist(), edges=q.edges.tolist(), exit=r.returncode,
                               printed=[int(c) for _, c in m], et=[e for e, _ in m])
                except subprocess.TimeoutExpired:
                    rec = dict(graph=dict(name=gname, scale=scale, edge_factor=ef, labels=nl, zipf_s=zs, seed=seed),
                               labels=q.labels.tolist(), edges=q.edges.tolist(), exit="timeout", printed=[], et=[])
                cases.append(rec)
                print(gname, k, dens, i, rec["exit"], rec["printed"], flush=True)
    with open(out, "w") as f:
        json.dump({"binary": "oracle/_ref/GEM_ic (in-core, built by oracle/ref/Makefile)", "threshold": 0,
                   "cases": cases}, f, indent=0)


if __name__ == "__main__":
    main()
