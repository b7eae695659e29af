"""Generates tests/golden/cases.json: small labelled graphs and queries with
expected embedding counts and embedding hashes.

Expected values come from two independent sources, neither of them the
backtracking oracle under test:
  * closed-form answers (complete graphs, cycles, stars, bipartite graphs);
  * exhaustive enumeration of every injective label-preserving map, written
    here in pure Python (itertools.permutations) for graphs of <= 12 vertices.
The embedding hash follows gem_embedding_hash (include/gem.h): splitmix64
finaliser of the sum of per-vertex terms, summed over embeddings mod 2^64.
Run: python tests/golden/make_golden.py
"""
import itertools
import json
import os
import random

M = (1 << 64) - 1


def mix64(x):
    x = (x + 0x9E3779B97F4A7C15) & M
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
    return x ^ (x >> 31)


def emb_hash(f):
    s = 0
    for u, v in enumerate(f):
        s = (s + mix64(v | (u << 32))) & M
    return mix64(s)


def enumerate_count(nv, edges, labels, qn, qedges, qlabels):
    adj = set()
    for a, b in edges:
        adj.add((a, b))
        adj.add((b, a))
    cnt, h = 0, 0
    for f in itertools.permutations(range(nv), qn):
        if any(labels[f[u]] != qlabels[u] for u in range(qn)):
            continue
        if all((f[a], f[b]) in adj for a, b in qedges):
            cnt += 1
            h = (h + emb_hash(f)) & M
    return cnt, h


def complete(n):
    return [(i, j) for i in range(n) for j in range(i + 1, n)]


def cycle(n):
    return [(i, (i + 1) % n) for i in range(n)]


def main():
    cases = []

    def add(name, nv, edges, labels, qn, qedges, qlabels, closed_form=None):
        c, h = enumerate_count(nv, edges, labels, qn, qedges, qlabels)
        if closed_form is not None:
            assert c == closed_form, (name, c, closed_form)
        cases.append(dict(name=name, nv=nv, edges=[list(e) for e in edges], labels=list(labels), qn=qn,
                          qedges=[list(e) for e in qedges], qlabels=list(qlabels), count=c, hash=str(h),
                          closed_form=closed_form))

    # closed forms (unlabelled = all labels 0)
    add("triangle_in_K4", 4, complete(4), [0] * 4, 3, cycle(3), [0] * 3, 4 * 6)
    add("triangle_in_K5", 5, complete(5), [0] * 5, 3, cycle(3), [0] * 3, 10 * 6)
    k33 = [(i, 3 + j) for i in range(3) for j in range(3)]
    add("C4_in_K33", 6, k33, [0] * 6, 4, cycle(4), [0] * 4, 9 * 8)
    add("triangle_in_K33", 6, k33, [0] * 6, 3, cycle(3), [0] * 3, 0)
    add("edge_in_C5", 5, cycle(5), [0] * 5, 2, [(0, 1)], [0, 0], 10)
    add("P3_in_K4", 4, complete(4), [0] * 4, 3, [(0, 1), (1, 2)], [0] * 3, 24)
    add("star3_in_K14", 5, [(0, i) for i in range(1, 5)], [0] * 5, 4, [(0, 1), (0, 2), (0, 3)], [0] * 4, 4 * 3 * 2)
    add("K4_in_K6", 6, complete(6), [0] * 6, 4, complete(4), [0] * 4, 6 * 5 * 4 * 3)
    add("single_vertex", 5, cycle(5), [0, 1, 0, 1, 2], 1, [], [1], 2)
    add("label_absent", 5, cycle(5), [0] * 5, 2, [(0, 1)], [0, 7], 0)
    # labelled: bipartite labels on K33 -> C4 with alternating labels
    add("C4_alt_labels_K33", 6, k33, [0, 0, 0, 1, 1, 1], 4, cycle(4), [0, 1, 0, 1], 9 * 4)
    # random labelled graphs, exhaustive enumeration
    rng = random.Random(0x474F4C44)
    for t in range(14):
        nv = rng.randint(6, 10)
        p = rng.choice([0.3, 0.45, 0.6])
        edges = [(i, j) for i in range(nv) for j in range(i + 1, nv) if rng.random() < p]
        L = rng.choice([1, 2, 3])
        labels = [rng.randrange(L) for _ in range(nv)]
        qn = rng.randint(2, min(5, nv))
        qedges = set()
        nbrs = {v: [b if a == v else a for a, b in edges if v in (a, b)] for v in range(nv)}
        start = rng.randrange(nv)
        walk = [start]
        cur = start
        for _ in range(200):
            if len(walk) == qn or not nbrs[cur]:
                break
            cur = rng.choice(nbrs[cur])
            if cur not in walk:
                walk.append(cur)
        if t % 2 == 0 and len(walk) == qn:
            # extracted from the graph (>= 1 match): induced edges, a few dropped
            for i in range(qn):
                for j in range(i + 1, qn):
                    if (min(walk[i], walk[j]), max(walk[i], walk[j])) in set(edges):
                        qedges.add((i, j))
            qlabels = [labels[v] for v in walk]
            # keep connectivity: only drop an edge if the rest stays connected
            for e in sorted(qedges):
                if rng.random() < 0.3:
                    rest = qedges - {e}
                    seen, stack = {0}, [0]
                    while stack:
                        x = stack.pop()
                        for a, b in rest:
                            y = b if a == x else (a if b == x else None)
                            if y is not None and y not in seen:
                                seen.add(y)
                                stack.append(y)
                    if len(seen) == qn:
                        qedges = rest
        else:
            # connected random query: spanning tree + extra edges
            for v in range(1, qn):
                qedges.add((rng.randrange(v), v))
            for i in range(qn):
                for j in range(i + 1, qn):
                    if rng.random() < 0.3:
                        qedges.add((i, j))
            qlabels = [rng.randrange(L) for _ in range(qn)]
        qedges = sorted(qedges)
        add(f"random_{t}", nv, edges, labels, qn, qedges, qlabels)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cases.json")
    with open(out, "w") as f:
        json.dump(cases, f, indent=0)
    print(f"wrote {len(cases)} cases to {out}")


if __name__ == "__main__":
    main()
