"""Nested-dissection ordering in the oracle (the rules hp_node_nd follows):
a permutation, separators that separate, far less fill than the natural
order on meshes, and the fill counter against a dense elimination."""
import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs


def _dense_fill(g, iperm):
    """Entries of L by explicit elimination of a dense boolean matrix (small n)."""
    n = g.nvtxs
    a = np.zeros((n, n), bool)
    for v in range(n):
        for u in g.adjncy[g.xadj[v]:g.xadj[v + 1]]:
            a[iperm[v], iperm[u]] = True
    np.fill_diagonal(a, True)
    nnz = 0
    for k in range(n):
        col = np.nonzero(a[k + 1:, k])[0] + k + 1
        nnz += 1 + col.size
        a[np.ix_(col, col)] = True
    return nnz


@pytest.mark.parametrize("seed", [1, 2])
def test_cholesky_nnz_matches_dense_elimination(seed):
    g = graphs.rmat(7, 4, seed=seed)
    rng = np.random.default_rng(seed)
    iperm = rng.permutation(g.nvtxs).astype(np.int32)
    assert oracle.cholesky_nnz(g, iperm) == _dense_fill(g, iperm)
    ident = np.arange(g.nvtxs, dtype=np.int32)
    assert oracle.cholesky_nnz(g, ident) == _dense_fill(g, ident)


@pytest.mark.parametrize("name", ["grid2d_64", "grid3d_14", "rmat12", "rgg4k"])
def test_nd_is_a_permutation_with_less_fill(name):
    g = {"grid2d_64": lambda: graphs.grid2d(64, 64),
         "grid3d_14": lambda: graphs.grid3d(14, 14, 14, seed=2, wmin=1, wmax=1),
         "rmat12": lambda: graphs.rmat(12, 8, seed=5),
         "rgg4k": lambda: graphs.rgg(4096, 10.0, seed=4)}[name]()
    oracle.set_threads(4)
    perm, iperm = oracle.node_nd(g)
    n = g.nvtxs
    assert np.array_equal(np.sort(iperm), np.arange(n))
    assert np.array_equal(perm[iperm], np.arange(n))
    nat = oracle.cholesky_nnz(g, np.arange(n, dtype=np.int32))
    nd = oracle.cholesky_nnz(g, iperm)
    if name.startswith("grid"):
        assert nd < 0.6 * nat, (nd, nat)
    else:
        assert nd <= nat
    # deterministic
    assert np.array_equal(oracle.node_nd(g)[1], iperm)


def test_nd_separator_separates():
    g = graphs.grid2d(40, 30)
    where = (np.arange(g.nvtxs) % 40 >= 17).astype(np.int32)   # a vertical cut
    side = oracle.nd_separator(g, where)
    assert set(np.unique(side)) <= {0, 1, 2}
    src = np.repeat(np.arange(g.nvtxs), np.diff(g.xadj))
    a, b = side[src], side[g.adjncy]
    assert not np.any((a == 0) & (b == 1)) and not np.any((a == 1) & (b == 0))
    assert (side == 2).sum() == 30   # one column of the grid


def test_nd_small_and_edgeless():
    g = graphs.grid2d(5, 5)                     # a leaf: minimum degree on the whole graph
    perm, iperm = oracle.node_nd(g)
    assert np.array_equal(np.sort(iperm), np.arange(25))
    assert iperm[0] == 0                         # a corner has the least degree and the lowest id
    e = graphs.Graph(np.zeros(301, np.int32), np.zeros(0, np.int32), np.ones(300, np.int32),
                     np.zeros(0, np.int32))
    assert np.array_equal(oracle.node_nd(e)[1], np.arange(300))
