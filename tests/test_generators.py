"""The oracle's seeded workload generators (used by the benchmark's reference
arm, which must not load libgem) give the same graphs and queries as
libgem's gem_hgraph_rmat / gem_hgraph_set_labels / gem_gen_queries."""
import numpy as np
import pytest

import gem_b200 as gem
import oracle


@pytest.mark.parametrize("scale,ef,nl,zs,seed", [(10, 8, 4, 0.0, 0x47454D0A), (12, 16, 16, 1.0, 0x47454D0C),
                                                 (13, 8, 32, 1.2, 0x1234), (16, 8, 8, 0.0, 0x47454D00 + 16)])
def test_graph_and_queries_equal_libgem(scale, ef, nl, zs, seed):
    og = oracle.set_labels(oracle.rmat(scale, ef, seed=seed), nl, zs, seed=seed ^ 0x4C)
    gg = gem.HostGraph.rmat(scale, ef, seed=seed).set_labels(nl, zs, seed=seed ^ 0x4C)
    off, nbr, lab = gg.arrays()
    assert np.array_equal(off, og.off) and np.array_equal(nbr, og.nbr) and np.array_equal(lab, og.lab)
    for k in (2, 4, 8, 12, 24, 32):
        for d in (gem.ANY, gem.SPARSE, gem.DENSE):
            a = oracle.gen_queries(og, k, d, 12, seed=0x51000 + k + 7 * d)
            b = gem.gen_queries(gg, k, d, 12, seed=0x51000 + k + 7 * d)
            for x, y in zip(a, b):
                assert np.array_equal(x.labels, y.labels) and np.array_equal(x.edges, y.edges), (k, d)


def test_bench_pools_equal_between_arms():
    """bench.py builds the reference arm's inputs with the oracle and its own
    with libgem: the config-3 mix and the config-1 pool must be the same
    queries, and both arms print the same config."""
    import bench
    og = oracle.set_labels(oracle.rmat(12, 8, seed=0x61), 16, 1.0, seed=0x62)
    gg = gem.HostGraph.rmat(12, 8, seed=0x61).set_labels(16, 1.0, seed=0x62)
    for a, b in ((bench.mix_pool(oracle, og, 60), bench.mix_pool(gem, gg, 60)),
                 (bench.config1_pool(oracle, og, 30), bench.config1_pool(gem, gg, 30))):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            assert np.array_equal(x.labels, y.labels) and np.array_equal(x.edges, y.edges)
    sizes = sorted({q.nv for q in bench.mix_pool(oracle, og, 60)})
    assert sizes == list(bench.MIX_SIZES)
    tune = bench.mix_pool(oracle, og, 60, seed=0x51083)
    main = bench.mix_pool(oracle, og, 60)
    assert not any(np.array_equal(x.edges, y.edges) and np.array_equal(x.labels, y.labels) and x.nv > 4
                   for x in tune for y in main)
    for w in ("rmat22-mix", "rmat16"):
        args = bench.parse_args(["--workload", w])
        assert bench.workload_config(w, args, 1) == bench.workload_config(w, args, 1)
