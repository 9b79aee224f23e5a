"""Nested-dissection ordering on the GPU (hp_node_nd, through the C ABI):
iperm bit-identical to the oracle's (ora_node_nd) on meshes, power-law and
geometric graphs, a graph with hubs, and the edge cases (a leaf-sized graph,
no edges, vertex weights); invalid input is rejected like a partition's."""
import numpy as np
import pytest

import hunyuansc25_b200 as hp
import oracle
from hunyuansc25_b200 import graphs
from hunyuansc25_b200._abi import HP_ERR_INVALID_GRAPH, default_options

pytestmark = pytest.mark.gpu

CASES = {
    "grid2d_100x80": lambda: graphs.grid2d(100, 80),
    "grid3d_20": lambda: graphs.grid3d(20, 20, 20, seed=2, wmin=1, wmax=1),
    "rmat12": lambda: graphs.rmat(12, 8, seed=5),
    "rgg14": lambda: graphs.rgg(1 << 14, 10.0, seed=4),
    "weighted_grid": lambda: graphs.grid2d(60, 50, seed=7, wmin=1, wmax=9),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_nd_equals_oracle(ctx, name):
    g = CASES[name]()
    if name == "weighted_grid":   # vertex weights take part in the separator partitions
        g = graphs.Graph(g.xadj, g.adjncy, (np.arange(g.nvtxs) % 5 + 1).astype(np.int32), g.adjwgt)
    perm_o, iperm_o = oracle.node_nd(g)
    perm, iperm = ctx.node_nd_graph(g)
    assert np.array_equal(iperm, iperm_o)
    assert np.array_equal(perm, perm_o)
    st = ctx.stats()
    assert st.nlevels >= 1 and st.kernel_launches > 0


def test_nd_large_mesh_fill(ctx):
    """A 64^3 mesh: equal to the oracle, and far less fill than the natural order."""
    g = graphs.grid3d(64, 64, 64, seed=2, wmin=1, wmax=1)
    _, iperm = ctx.node_nd_graph(g)
    _, iperm_o = oracle.node_nd(g)
    assert np.array_equal(iperm, iperm_o)
    nat = oracle.cholesky_nnz(g, np.arange(g.nvtxs, dtype=np.int32))
    assert oracle.cholesky_nnz(g, iperm) < 0.25 * nat


def test_nd_edge_cases(ctx):
    small = graphs.grid2d(9, 9)   # one leaf
    assert np.array_equal(ctx.node_nd_graph(small)[1], oracle.node_nd(small)[1])
    e = graphs.Graph(np.zeros(501, np.int32), np.zeros(0, np.int32), np.ones(500, np.int32), np.zeros(0, np.int32))
    assert np.array_equal(ctx.node_nd_graph(e)[1], np.arange(500))
    one = graphs.Graph(np.array([0, 0], np.int32), np.zeros(0, np.int32), np.ones(1, np.int32), np.zeros(0, np.int32))
    assert np.array_equal(ctx.node_nd_graph(one)[1], [0])
    # a star with a ring: hub rows and a separator of one vertex
    n = 3000
    src = [0] * (n - 1) + list(range(1, n - 1))
    dst = list(range(1, n)) + list(range(2, n))
    s = np.array(src + dst); d = np.array(dst + src)
    o = np.lexsort((d, s))
    xadj = np.zeros(n + 1, np.int64)
    np.add.at(xadj, s + 1, 1)
    star = graphs.Graph(np.cumsum(xadj).astype(np.int32), d[o].astype(np.int32), np.ones(n, np.int32),
                        np.ones(len(s), np.int32))
    assert np.array_equal(ctx.node_nd_graph(star)[1], oracle.node_nd(star)[1])


def test_nd_invalid_input(ctx):
    xadj = np.array([0, 1, 2], np.int32)
    with pytest.raises(hp.HpError) as e:
        ctx.node_nd(xadj, np.array([0, 0], np.int32))   # self loop
    assert e.value.code == HP_ERR_INVALID_GRAPH
    g = graphs.grid2d(30, 30)
    assert np.array_equal(ctx.node_nd_graph(g)[1], oracle.node_nd(g)[1])   # still usable
