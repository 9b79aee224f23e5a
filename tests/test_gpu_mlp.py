"""Learned move proposals: device training kernels against the CPU oracle
(and reproducible), tensor-core inference against FP32, the move log, a
learned partition that stays exact (cut recomputed, balance honoured) and
deterministic, and what the committed network gains over the plain refiner."""
import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs, learn
from hunyuansc25_b200._abi import HP_MLP_NPARAM, default_options

pytestmark = pytest.mark.gpu


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.6, size=(n, 8)).astype(np.float32)
    y = ((x[:, 0] + 0.5 * x[:, 5] - 0.3 * x[:, 1]) > 0).astype(np.float32)
    return x, y


def test_gradient_matches_oracle(ctx):
    import torch
    x, y = _data(5000, 1)
    p = learn.init_params(3)
    p[256:288] = 0.05   # nonzero biases exercise their gradients
    ctx.mlp_set_params(p)
    loss, g = ctx.mlp_loss_grad(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    oloss, og = oracle.mlp_loss_grad(p, x, y)
    # FP32 device sums (fixed order) vs double-accumulated CPU: rel-err <= 1e-3
    assert abs(loss - oloss) <= 1e-3 * max(1.0, abs(oloss))
    scale = np.abs(og).max()
    assert np.max(np.abs(g - og)) <= 1e-3 * scale, (np.max(np.abs(g - og)), scale)


def test_inference_tensor_cores_vs_fp32(ctx):
    import torch
    x, _ = _data(10007, 2)
    p = learn.init_params(4)
    ctx.mlp_set_params(p)
    xt = torch.from_numpy(x).cuda()
    ref = oracle.mlp_forward(p, x)
    fp32 = ctx.mlp_infer(xt, tensor_cores=False).cpu().numpy()
    bf16 = ctx.mlp_infer(xt, tensor_cores=True).cpu().numpy()
    assert np.allclose(fp32, ref, rtol=1e-4, atol=1e-4)
    # BF16 operands (8-bit mantissa), FP32 accumulation: |err| <= 0.03 + 0.03 |y|
    err = np.abs(bf16 - ref)
    assert np.all(err <= 0.03 + 0.03 * np.abs(ref)), err.max()
    assert np.mean(np.sign(bf16) == np.sign(ref)) > 0.99


def test_training_lowers_loss(ctx):
    import torch
    x, y = _data(40000, 5)
    p0 = learn.init_params(7)
    ctx.mlp_set_params(p0)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    l0, _ = ctx.mlp_loss_grad(xt, yt)
    params, losses = learn.train(ctx, x, y, epochs=8, batch=2048, lr=3e-3, seed=7, params=p0)
    l1, _ = ctx.mlp_loss_grad(xt, yt)
    assert l1 < 0.5 * l0
    acc = np.mean((oracle.mlp_forward(params, x) > 0) == (y > 0.5))
    assert acc > 0.95


def test_training_is_reproducible(ctx):
    """Gradients are summed in a fixed order (no float atomics): the same data,
    initial weights and shuffling seed give bit-identical weights."""
    x, y = _data(20000, 9)
    p0 = learn.init_params(11)
    runs = []
    for _ in range(2):
        ctx.mlp_set_params(p0)
        params, losses = learn.train(ctx, x, y, epochs=3, batch=4096, lr=3e-3, seed=5, params=p0)
        runs.append((params.copy(), list(losses)))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_move_log_does_not_change_the_partition(ctx):
    g = graphs.rmat(13, 16, seed=11)
    plain_part, plain_cut = ctx.partition_graph(g, 64)
    ctx.movelog_enable(1 << 20)
    part, cut = ctx.partition_graph(g, 64, options=default_options(learned=2))
    assert cut == plain_cut and np.array_equal(part, plain_part)
    x, y = ctx.movelog_fetch()
    assert x.shape[0] > 100 and np.all(np.isfinite(x))
    assert set(np.unique(y)).issubset({0.0, 1.0})
    assert 0.0 < y.mean() < 1.0
    ctx.movelog_enable(0)


def test_learned_partition_exact_and_deterministic(ctx):
    g = graphs.rmat(13, 16, seed=21)
    ctx.movelog_enable(1 << 21)
    ctx.partition_graph(graphs.rmat(12, 16, seed=22), 64, options=default_options(learned=2))
    x, y = ctx.movelog_fetch()
    ctx.movelog_enable(0)
    params, _ = learn.train(ctx, x, y, epochs=4, batch=2048, seed=1)
    thr, _ = learn.pick_threshold(ctx, x, y)
    ctx.mlp_set_params(params, thr)
    plain_part, plain_cut = ctx.partition_graph(g, 64)
    lopt = default_options(learned=1)
    a_part, a_cut = ctx.partition_graph(g, 64, options=lopt)
    st = ctx.stats()
    b_part, b_cut = ctx.partition_graph(g, 64, options=lopt)
    assert a_cut == b_cut and np.array_equal(a_part, b_part)
    assert a_cut == oracle.edgecut(g, a_part)           # exact int64 cut
    assert st.max_excess <= 0                            # balance bound honoured exactly
    assert a_cut <= 1.10 * plain_cut
    # the CUDA-graph pass loop (both LP kernels captured, gated on the device by
    # the learned flag) gives the same partition as the eager loop
    e_part, e_cut = ctx.partition_graph(g, 64, options=default_options(learned=1, eager=1))
    assert e_cut == a_cut and np.array_equal(e_part, a_part)


def test_learned_gain_over_plain(ctx):
    """What the committed network gains on a mid-size R-MAT (scale 18, k = 256):
    the same balanced partition quality (cut within 1 % of the plain refiner's,
    measured 0.4 % lower) for a fraction of the refinement work -- the moves
    applied and the gain rows rebuilt, counted on the device -- and less device
    time (measured 1.12x; asserted >= 1.05x, best of three runs each)."""
    g = graphs.rmat(18, 16, seed=3, wmin=1, wmax=100)
    params, thr, _ = learn.load_params()
    ctx.mlp_set_params(params, thr)
    res = {}
    for mode in (0, 1):
        ms = []
        for it in range(4):
            part, cut = ctx.partition_graph(g, 256, 1.03, options=default_options(learned=mode))
            st = ctx.stats()
            if it:
                ms.append(st.ms_total)
        assert st.max_excess <= 0
        ctx.partition_graph(g, 256, 1.03, options=default_options(learned=mode, profile=1, eager=1))
        pst = ctx.stats()
        res[mode] = dict(ms=min(ms), cut=cut, apply=pst.prof_bytes[8], rebuild=pst.prof_bytes[4])
    plain, learned = res[0], res[1]
    assert learned["cut"] <= 1.01 * plain["cut"]
    assert learned["apply"] <= 0.25 * plain["apply"]
    assert learned["rebuild"] <= 0.5 * plain["rebuild"]
    assert plain["ms"] / learned["ms"] >= 1.05, (plain["ms"], learned["ms"])


@pytest.mark.parametrize("name", ["rmat14", "rmat13_k64", "rmat15_k1024"])
def test_judged_learned_passes(ctx, name):
    """learned = 3: every learned LP pass is judged by the plain refiner on the
    same state (exact cut decrease of both move sets from one afterburner walk
    and one pass over the moved rows).  The judge's sum over the learned moves
    is checked on the device against the applied pass's exact cut change (a
    mismatch fails the call with HP_ERR_INTERNAL); results are deterministic and
    the same in the CUDA-graph loop, the eager loop and the one-CTA small-level
    loop, and the partition is balanced with its exact cut."""
    if name == "rmat14":
        g, k = graphs.rmat(14, 16, seed=3, wmin=1, wmax=100), 256
    elif name == "rmat13_k64":
        g, k = graphs.rmat(13, 16, seed=8, wmin=1, wmax=100), 64
    else:
        g, k = graphs.rmat(15, 16, seed=9, wmin=1, wmax=100), 1024
    params, thr, _ = learn.load_params()
    ctx.mlp_set_params(params, thr)
    jopt = default_options(learned=3)
    a_part, a_cut = ctx.partition_graph(g, k, options=jopt)
    st = ctx.stats()
    assert st.max_excess <= 0
    assert a_cut == oracle.edgecut(g, a_part)
    b_part, b_cut = ctx.partition_graph(g, k, options=jopt)
    assert b_cut == a_cut and np.array_equal(b_part, a_part)
    e_part, e_cut = ctx.partition_graph(g, k, options=default_options(learned=3, eager=1))
    assert e_cut == a_cut and np.array_equal(e_part, a_part)
    ctx.set_tuning(small_level_n=0)
    try:
        m_part, m_cut = ctx.partition_graph(g, k, options=jopt)
    finally:
        ctx.set_tuning(None)
    assert m_cut == a_cut and np.array_equal(m_part, a_part)


def test_learned_mode_runs_plain_on_meshes(ctx):
    """The learned proposals apply to inputs whose largest degree is at least 16x
    the mean (the power-law graphs the network is validated on); a mesh or a
    geometric graph is refined by the plain rule, so learned = 1 and 3 give the
    plain partition bit for bit, while a power-law graph does not."""
    params, thr, _ = learn.load_params()
    ctx.mlp_set_params(params, thr)
    for g, k in ((graphs.grid3d(32, 32, 32, seed=2, wmin=1, wmax=10), 64), (graphs.rgg(1 << 16, 12.0, seed=4), 256)):
        p0, c0 = ctx.partition_graph(g, k, options=default_options(learned=0))
        for mode in (1, 3):
            p1, c1 = ctx.partition_graph(g, k, options=default_options(learned=mode))
            assert c1 == c0 and np.array_equal(p1, p0)
    g = graphs.rmat(14, 16, seed=3, wmin=1, wmax=100)
    p0, c0 = ctx.partition_graph(g, 256, options=default_options(learned=0))
    p1, c1 = ctx.partition_graph(g, 256, options=default_options(learned=1))
    assert not np.array_equal(p1, p0)
