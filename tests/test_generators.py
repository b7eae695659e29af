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
