"""Synthetic workload generators: structure, symmetry and weight hashing."""
import numpy as np
import pytest

from hunyuansc25_b200 import graphs


def check_simple_symmetric(g):
    n = g.nvtxs
    assert g.xadj[0] == 0 and g.xadj[-1] == g.nedges
    assert np.all(np.diff(g.xadj) >= 0)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(g.xadj))
    dst = g.adjncy.astype(np.int64)
    assert np.all((dst >= 0) & (dst < n))
    assert not np.any(src == dst), "self loop"
    key = src * n + dst
    # rows sorted strictly ascending -> no duplicates
    for v in range(0, n, max(1, n // 200)):
        r = g.adjncy[g.xadj[v]:g.xadj[v + 1]]
        assert np.all(np.diff(r) > 0)
    rkey = dst * n + src
    o1 = np.argsort(key)
    o2 = np.argsort(rkey)
    assert np.array_equal(key[o1], rkey[o2]), "not symmetric"
    assert np.array_equal(g.adjwgt[o1], g.adjwgt[o2]), "weights not symmetric"
    assert np.all(g.adjwgt > 0) and np.all(g.vwgt == 1)


def test_grid2d_shape():
    g = graphs.config_grid2d()
    assert g.nvtxs == 65536 and g.nedges == 2 * 130560
    assert np.all(g.adjwgt == 1)
    check_simple_symmetric(g)


def test_grid3d_small():
    g = graphs.grid3d(9, 7, 5, seed=2, wmin=1, wmax=10)
    assert g.nvtxs == 315
    assert g.nedges == 2 * (8 * 7 * 5 + 9 * 6 * 5 + 9 * 7 * 4)
    assert g.adjwgt.min() >= 1 and g.adjwgt.max() <= 10
    check_simple_symmetric(g)


def test_grid3d_config_counts():
    # 128^3: 2,097,152 vertices, 6,242,304 undirected edges
    n = 128 ** 3
    m = 3 * 127 * 128 * 128
    assert n == 2097152 and m == 6242304


def test_rmat_small():
    g = graphs.rmat(10, 8, seed=3, wmin=1, wmax=100)
    assert g.nvtxs == 1024
    check_simple_symmetric(g)
    assert g.adjwgt.min() >= 1 and g.adjwgt.max() <= 100


def test_rmat_limit():
    g = graphs.rmat(11, 8, seed=7, wmin=1, wmax=100, nvtxs_limit=1500)
    assert g.nvtxs == 1500
    check_simple_symmetric(g)


def test_rgg_small():
    g = graphs.rgg(4000, 12.0, seed=4)
    check_simple_symmetric(g)
    assert g.adjwgt.min() >= 1 and g.adjwgt.max() <= 1001
    assert 9 < g.nedges / g.nvtxs < 13


def test_weight_hash_symmetric_and_seeded():
    a = graphs.edge_weight(5, 3, 9, 1, 100)
    b = graphs.edge_weight(5, 9, 3, 1, 100)
    c = graphs.edge_weight(6, 3, 9, 1, 100)
    assert a == b
    assert 1 <= a <= 100
    vals = {graphs.edge_weight(s, 3, 9, 1, 100) for s in range(40)}
    assert len(vals) > 10
    assert c in vals


def test_generators_deterministic():
    g1 = graphs.rmat(9, 4, seed=11)
    g2 = graphs.rmat(9, 4, seed=11)
    assert np.array_equal(g1.adjncy, g2.adjncy) and np.array_equal(g1.adjwgt, g2.adjwgt)


def test_batch_specs():
    specs = graphs.batch_specs(64, seed=5)
    assert len(specs) == 64
    for kind, n, k in specs:
        assert kind in ("grid2d", "rmat")
        assert 1000 <= n <= 200000
        assert k in (2, 4, 8, 16, 32, 64)
