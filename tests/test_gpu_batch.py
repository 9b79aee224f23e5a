"""Batched partition of many independent graphs (hp_partition_batch): every
graph's result equals its single-call result (and therefore the oracle's)."""
import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs

pytestmark = pytest.mark.gpu


def test_batch_equals_single_calls(ctx):
    specs = graphs.batch_specs(24, seed=5, nmin=300, nmax=6000)
    gs = [graphs.batch_graph(kind, n, seed=100 + i) for i, (kind, n, k) in enumerate(specs)]
    ks = [k for _, _, k in specs]
    parts, cuts = ctx.partition_batch(gs, ks, 1.03)
    for g, k, p, c in zip(gs, ks, parts, cuts):
        sp, sc = ctx.partition_graph(g, k, 1.03)
        assert c == sc
        assert np.array_equal(p, sp)
        assert c == oracle.edgecut(g, p)
    st = ctx.stats()
    assert st.kernel_launches > 0


def test_batch_oracle_parity_small(ctx):
    gs = [graphs.grid2d(30 + i, 20, seed=i, wmin=1, wmax=9) for i in range(6)]
    ks = [2, 3, 4, 5, 6, 7]
    parts, cuts = ctx.partition_batch(gs, ks, 1.03)
    for g, k, p, c in zip(gs, ks, parts, cuts):
        op, oc, _ = oracle.partition(g, k, 1.03)
        assert oc == c and np.array_equal(op, p)


def test_batch_error_reported(ctx):
    import hunyuansc25_b200 as hp
    good = graphs.grid2d(10, 10)
    bad = graphs.Graph(np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32),
                       np.ones(2, np.int32), np.ones(2, np.int32))
    with pytest.raises(hp.HpError):
        ctx.partition_batch([good, bad], [2, 2], 1.03)
    parts, cuts = ctx.partition_batch([good], [2], 1.03)
    assert cuts[0] == oracle.edgecut(good, parts[0])


def test_prepared_batch_matches_batch_call(ctx):
    gs = [graphs.batch_graph("rmat" if i % 2 else "grid2d", 2000 + 500 * i, seed=300 + i) for i in range(5)]
    ks = [2, 4, 8, 16, 32]
    parts, cuts = ctx.partition_batch(gs, ks, 1.03)
    b = ctx.prepare_batch(gs, ks, 1.03)
    for _ in range(2):   # the prepared arrays serve repeated calls
        p2, c2 = ctx.partition_prepared(b)
        assert [int(x) for x in c2] == [int(x) for x in cuts]
        for a, q in zip(parts, p2):
            assert np.array_equal(a, q)
