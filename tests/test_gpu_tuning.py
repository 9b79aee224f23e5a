"""Kernel tuning on the GPU: extreme row-class bounds, grid sizes and bitmap
layouts route rows through other kernels, and every level must still equal
the oracle bit for bit; invalid tunings are refused; the autotuner keeps
partitions identical."""
import json

import numpy as np
import pytest

import hunyuansc25_b200 as hp
from hunyuansc25_b200 import graphs, tune
from hunyuansc25_b200._abi import HP_ERR_INVALID_ARG, TUNING_DEFAULTS

from test_gpu_parity import compare_runs

pytestmark = pytest.mark.gpu

# every row past a few entries on the warp, CTA and hub paths; levels up to
# 32768 vertices refined by the one-CTA pass loop
SMALL_CLASSES = dict(match_warp_deg=4, match_cta_deg=24, contract_thread_row=8, contract_warp_row=16,
                     contract_cta_row=48, gain_thread_deg=8, gain_hub_deg=24, warp_dense_k=0,
                     grid_ctas_per_sm=1, dense_sparse_ratio=1, small_level_n=32768, chunk_deg=8,
                     trial_cta_n=1, contract_smem_cn=49152, small_match_n=8192, contract_hybrid=1,
                     apply_chunk_deg=8)
# the largest per-thread and warp classes, many CTAs, every level on the
# multi-kernel pass loop, launched pass by pass without programmatic dependent
# launch
LARGE_CLASSES = dict(match_warp_deg=256, match_cta_deg=1 << 24, contract_thread_row=32, contract_warp_row=256,
                     contract_cta_row=4096, gain_thread_deg=32, gain_hub_deg=1 << 24, warp_dense_k=1024,
                     grid_ctas_per_sm=32, dense_sparse_ratio=4096, small_level_n=0, chunk_deg=1 << 24,
                     trial_cta_n=1 << 24, contract_smem_cn=0, small_match_n=0, contract_hybrid=0,
                     apply_chunk_deg=1 << 24, pdl=0, graph_passes=0)
MIXED = dict(match_warp_deg=16, match_cta_deg=256, contract_thread_row=16, contract_warp_row=64,
             contract_cta_row=512, gain_thread_deg=16, gain_hub_deg=512, warp_dense_k=256, grid_ctas_per_sm=3,
             dense_sparse_ratio=2, small_level_n=4096, chunk_deg=96, trial_cta_n=200,
             contract_smem_cn=3000, small_match_n=2000, apply_chunk_deg=64, pdl=0)


def hub_graph(n=20000):
    """A star plus a ring: one row of n-1 entries (the dense contraction path)."""
    src = [0] * (n - 1) + list(range(1, n - 1))
    dst = list(range(1, n)) + list(range(2, n))
    e = np.array(src + dst, np.int64), np.array(dst + src, np.int64)
    order = np.lexsort((e[1], e[0]))
    s, d = e[0][order], e[1][order]
    xadj = np.zeros(n + 1, np.int32)
    np.add.at(xadj, s + 1, 1)
    xadj = np.cumsum(xadj).astype(np.int32)
    w = np.array([graphs.edge_weight(1, int(a), int(b), 1, 50) for a, b in zip(s, d)], np.int32)
    return graphs.Graph(xadj, d.astype(np.int32), np.ones(n, np.int32), w)


CASES = {
    "rmat13_hubs": lambda: (graphs.rmat(13, 16, seed=3, wmin=1, wmax=100), 64, 1.03),
    "grid3d_24": lambda: (graphs.grid3d(24, 24, 24, seed=2, wmin=1, wmax=10), 32, 1.03),
    "rgg16_k1024": lambda: (graphs.rgg(1 << 16, 12.0, seed=4), 1024, 1.05),
    "hub20k": lambda: (hub_graph(), 16, 1.03),
}


def make_case(name):
    return CASES[name]()


@pytest.fixture(scope="module")
def tctx():
    c = hp.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("tuning", [SMALL_CLASSES, LARGE_CLASSES, MIXED], ids=["small", "large", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tuned_levels_equal_oracle(tctx, name, tuning):
    g, k, ub = make_case(name)
    tctx.set_tuning(tuning)
    try:
        assert tctx.get_tuning() == dict(TUNING_DEFAULTS, **tuning)
        compare_runs(tctx, g, k, ub)
    finally:
        tctx.set_tuning(None)


@pytest.mark.parametrize("tuning", [SMALL_CLASSES, MIXED], ids=["small", "mixed"])
def test_tuned_learned_and_eager_equal_default(tctx, tuning):
    from hunyuansc25_b200 import learn
    g, k, ub = make_case("rmat13_hubs")
    params, thr, _ = learn.load_params()
    tctx.mlp_set_params(params, thr)
    for kw in (dict(learned=1), dict(eager=1)):
        opt = hp.default_options(**kw)
        tctx.set_tuning(None)
        p0, c0 = tctx.partition_graph(g, k, ub, options=opt)
        tctx.set_tuning(tuning)
        try:
            p1, c1 = tctx.partition_graph(g, k, ub, options=opt)
        finally:
            tctx.set_tuning(None)
        assert c0 == c1 and np.array_equal(p0, p1), kw


def test_batch_workers_inherit_tuning(tctx):
    gs = [graphs.batch_graph("rmat" if i % 2 else "grid2d", 3000 + 700 * i, seed=100 + i) for i in range(6)]
    ks = [4, 8, 16, 4, 8, 32]
    tctx.set_tuning(SMALL_CLASSES)
    try:
        parts, cuts = tctx.partition_batch(gs, ks, 1.03)
        assert tctx.get_tuning() == dict(TUNING_DEFAULTS, **SMALL_CLASSES)
    finally:
        tctx.set_tuning(None)
    for g, k, p, c in zip(gs, ks, parts, cuts):
        p0, c0 = tctx.partition_graph(g, k, 1.03)
        assert c0 == c and np.array_equal(p0, p)


@pytest.mark.parametrize("field,value", [("match_warp_deg", 2), ("contract_warp_row", 300),
                                         ("contract_cta_row", 8), ("warp_dense_k", 2048),
                                         ("grid_ctas_per_sm", 0)])
def test_invalid_tuning_refused(tctx, field, value):
    before = tctx.get_tuning()
    with pytest.raises(hp.HpError) as e:
        tctx.set_tuning({field: value})
    assert e.value.code == HP_ERR_INVALID_ARG
    assert tctx.get_tuning() == before


def test_autotune_small_space(tctx, tmp_path):
    g, k, ub = make_case("rmat13_hubs")
    space = {"match_warp_deg": [16, 32], "gain_thread_deg": [16, 32], "grid_ctas_per_sm": [4, 8]}
    best, rep = tune.autotune(tctx, g, k, ub, reps=1, sweeps=1, confirm=1, space=space)
    assert rep["identical_partitions"]
    assert rep["evaluations"] >= 1 + 3
    for f, v in best.items():
        assert v in space.get(f, [TUNING_DEFAULTS[f]])
    p = tmp_path / "rmat13.json"
    tune.write_tuning_file(str(p), best, **rep)
    t = tctx.load_tuning(str(p))
    assert t == best == tctx.get_tuning()
    assert json.loads(p.read_text())["tuning"] == best
    tctx.set_tuning(None)
