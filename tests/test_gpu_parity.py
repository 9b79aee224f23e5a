"""CUDA path vs the CPU oracle, through the C ABI: every level of the V-cycle
(coarse CSR, vertex/edge weights, matching, cmap, initial and projected
partitions, refined partitions, cuts) must be bit-identical."""
import ctypes as C
import os
import time

import numpy as np
import pytest

import hunyuansc25_b200 as hp
import oracle
from hunyuansc25_b200 import graphs
from hunyuansc25_b200._abi import (HP_ERR_INVALID_ARG, HP_ERR_INVALID_GRAPH, HP_ERR_NOMEM, HP_ERR_TIMEOUT,
                                   HP_ERR_UNSUPPORTED, default_options)

pytestmark = pytest.mark.gpu

NAMES = ["xadj", "adjncy", "adjwgt", "vwgt", "match", "cmap", "where_start", "where_final"]


def compare_runs(ctx, g, k, ub=1.03, tpwgts=None, **optkw):
    opt = default_options(trace=1, **optkw)
    oracle.set_threads(os.cpu_count() or 1)
    part_o, cut_o, tr = oracle.partition(g, k, ub, tpwgts=tpwgts, opt=opt, trace=True)
    part_g, cut_g = ctx.partition_graph(g, k, ub, tpwgts=tpwgts, options=opt)
    L = tr.nlevels
    assert ctx.trace_nlevels == L, (ctx.trace_nlevels, L)
    for l in reversed(range(L)):       # coarsest first: the first mismatch is the cause
        for what, name in enumerate(NAMES):
            a = tr.array(l, what)
            b = ctx.trace_array(l, what)
            if a is None:
                continue
            assert b is not None, f"level {l} {name} missing on GPU"
            if not np.array_equal(a, b):
                bad = np.nonzero(a != b)[0]
                raise AssertionError(f"level {l} {name}: {bad.size} entries differ, first at {bad[0]} "
                                     f"(oracle {a[bad[0]]}, gpu {b[bad[0]]})")
        assert ctx.trace_level(l) == tr.level(l), f"level {l} sizes/cuts differ"
    assert np.array_equal(part_o, part_g)
    assert cut_o == cut_g
    assert cut_g == oracle.edgecut(g, part_g)
    st = ctx.stats()
    assert st.edgecut == cut_g
    return part_g, cut_g, st


def test_grid2d_256_k8(ctx):
    g = graphs.config_grid2d()
    part, cut, st = compare_runs(ctx, g, 8, coarsen_to=160)
    assert st.max_excess <= 0


def test_grid2d_reference_threshold(ctx):
    compare_runs(ctx, graphs.config_grid2d(), 8)


def test_grid3d_32_k64(ctx):
    compare_runs(ctx, graphs.grid3d(32, 32, 32, seed=2, wmin=1, wmax=10), 64)


def test_rmat_s14_k256(ctx):
    compare_runs(ctx, graphs.rmat(14, 16, seed=3, wmin=1, wmax=100), 256)


def test_rmat_s12_unit(ctx):
    compare_runs(ctx, graphs.rmat(12, 16, seed=9, wmin=1, wmax=1), 32)


def test_rgg_k1024(ctx):
    compare_runs(ctx, graphs.rgg(1 << 16, 12.0, seed=4), 1024, ub=1.05)


def test_odd_k_and_tpwgts(ctx):
    g = graphs.grid2d(90, 70, seed=6, wmin=1, wmax=5)
    compare_runs(ctx, g, 7)
    tp = np.array([0.3, 0.2, 0.2, 0.1, 0.1, 0.05, 0.05], np.float32)
    compare_runs(ctx, g, 7, tpwgts=tp)


def test_seed_and_options(ctx):
    g = graphs.grid3d(20, 20, 20, seed=2, wmin=1, wmax=10)
    compare_runs(ctx, g, 16, seed=12345, match_rounds=3, refine_patience=2, init_starts=32, fm_passes=4)


def test_hub_graph_xl_rows(ctx):
    # a star plus a ring: one row far above the block-sort capacity
    n = 20000
    src = [0] * (n - 1) + list(range(1, n - 1))
    dst = list(range(1, n)) + list(range(2, n))
    e = np.array(src + dst, np.int64), np.array(dst + src, np.int64)
    order = np.lexsort((e[1], e[0]))
    s, d = e[0][order], e[1][order]
    xadj = np.zeros(n + 1, np.int32)
    np.add.at(xadj, s + 1, 1)
    xadj = np.cumsum(xadj).astype(np.int32)
    w = np.array([graphs.edge_weight(1, int(a), int(b), 1, 50) for a, b in zip(s, d)], np.int32)
    g = graphs.Graph(xadj, d.astype(np.int32), np.ones(n, np.int32), w)
    compare_runs(ctx, g, 8)


def test_full_grid3d_128_k64(ctx):
    """The 128^3 workload at full size: bit-identical to the oracle."""
    g = graphs.config_grid3d()
    part, cut, st = compare_runs(ctx, g, 64)
    assert st.max_excess <= 0
    assert part.min() >= 0 and part.max() < 64


def test_eager_passes_match_oracle(ctx):
    """The eager pass loop (one launch per kernel, a host read per pass) against
    the oracle, on the graphs the graph-mode tests above use; every level on the
    multi-kernel passes (the one-CTA small-level loop off)."""
    ctx.set_tuning(small_level_n=0)
    try:
        compare_runs(ctx, graphs.config_grid2d(), 8, coarsen_to=160, eager=1)
        compare_runs(ctx, graphs.rmat(14, 16, seed=3, wmin=1, wmax=100), 256, eager=1)
    finally:
        ctx.set_tuning(None)


@pytest.mark.parametrize("name", ["grid3d_48", "rmat13_hubs", "rgg17", "star"])
def test_graph_loop_equals_eager_loop(ctx, name):
    """CUDA-graph pass loop (device-side WHILE/SWITCH control, the one-CTA loop
    on the small levels) and the eager multi-kernel loop on every level give the
    same partition, cut and pass count."""
    if name == "grid3d_48":
        g, k = graphs.grid3d(48, 48, 48, seed=2, wmin=1, wmax=10), 64
    elif name == "rmat13_hubs":
        g, k = graphs.rmat(13, 16, seed=5, wmin=1, wmax=100), 128
    elif name == "rgg17":
        g, k = graphs.rgg(1 << 17, 12.0, seed=4), 512
    else:
        n = 20001
        xadj = np.zeros(n + 1, np.int32)
        xadj[1] = n - 1
        xadj[2:] = n - 1 + np.arange(1, n)
        adj = np.concatenate([np.arange(1, n), np.zeros(n - 1)]).astype(np.int32)
        g = graphs.Graph(xadj, adj, np.ones(n, np.int32), np.ones(2 * (n - 1), np.int32), "star")
        k = 16
    ctx.set_tuning(small_level_n=0)
    try:
        pe, ce = ctx.partition_graph(g, k, options=default_options(eager=1))
    finally:
        ctx.set_tuning(None)
    se = ctx.stats()
    pg, cg = ctx.partition_graph(g, k, options=default_options(eager=0))
    sg = ctx.stats()
    assert ce == cg and np.array_equal(pe, pg)
    assert se.refine_passes == sg.refine_passes
    assert sg.max_excess == se.max_excess


def test_deterministic_repeat(ctx):
    g = graphs.rmat(13, 16, seed=3)
    a = ctx.partition_graph(g, 64)
    b = ctx.partition_graph(g, 64)
    assert np.array_equal(a[0], b[0]) and a[1] == b[1]


def test_edge_cases(ctx):
    # empty graph
    part, cut = ctx.partition(np.zeros(1, np.int32), np.zeros(0, np.int32), 4)
    assert part.shape == (0,) and cut == 0
    # single vertex, k > n, k = 1
    g = graphs.grid2d(1, 1)
    part, cut = ctx.partition_graph(g, 4)
    assert cut == 0 and part.shape == (1,)
    g = graphs.grid2d(6, 6)
    part, cut = ctx.partition_graph(g, 1)
    assert cut == 0 and np.all(part == 0)
    compare_runs(ctx, g, 40)
    # isolated vertices + two components
    xadj = np.array([0, 1, 2, 2, 2, 4, 5, 6], np.int32)
    adj = np.array([1, 0, 5, 6, 4, 4], np.int32)
    gg = graphs.Graph(xadj, adj, np.ones(7, np.int32), np.ones(6, np.int32))
    compare_runs(ctx, gg, 2)
    compare_runs(ctx, gg, 3)


def mixed_matching_graph(leaves=400, isolated=200, tri=1000):
    """A star, isolated vertices and triangles weighted 3/2/1: the handshake
    rounds match the hub with one leaf and two vertices of each triangle; the
    other leaves pair through the hub (two-hop); the isolated vertices pair in
    id order; the third vertices of the triangles are forced into pairs."""
    n = 1 + leaves + isolated + 3 * tri
    rows = [[] for _ in range(n)]

    def edge(a, b, w):
        rows[a].append((b, w))
        rows[b].append((a, w))
    for i in range(1, leaves + 1):
        edge(0, i, 1)
    base = 1 + leaves + isolated
    for t in range(tri):
        a = base + 3 * t
        edge(a, a + 1, 3)
        edge(a + 1, a + 2, 2)
        edge(a, a + 2, 1)
    xadj = np.zeros(n + 1, np.int32)
    adj, w = [], []
    for v in range(n):
        r = sorted(rows[v])
        xadj[v + 1] = xadj[v] + len(r)
        adj += [u for u, _ in r]
        w += [x for _, x in r]
    return graphs.Graph(xadj, np.array(adj, np.int32), np.ones(n, np.int32), np.array(w, np.int32), "mixed")


@pytest.mark.parametrize("small_match_n", [4096, 0], ids=["one_cta", "multi_kernel"])
def test_matching_fallbacks(ctx, small_match_n):
    g = mixed_matching_graph()
    n = len(g.xadj) - 1
    _, _, tr = oracle.partition(g, 4, 1.03, opt=default_options(trace=1), trace=True)
    m = tr.array(0, 4)
    v = np.arange(n)
    pair = m > v
    leaf = (v >= 1) & (v <= 400)
    iso = (v >= 401) & (v <= 600)
    # the level-0 matching of this graph takes every fallback
    assert np.sum(pair & leaf & leaf[m]) == 199
    assert np.sum(pair & iso & iso[m]) == 100
    assert np.sum(pair & (v >= 601) & (m - v >= 3)) == 499   # forced: third vertices
    assert np.sum(pair & leaf & (m >= 601)) == 1             # forced: the last leaf
    ctx.set_tuning(small_match_n=small_match_n)
    try:
        compare_runs(ctx, g, 4)
        compare_runs(ctx, g, 64)
    finally:
        ctx.set_tuning()


def test_bounded_wait_expiry(ctx):
    """The failure path of the device waits: the scans' look-back wait on a flag
    that nothing sets gives up after its spin limit, the call reports
    HP_ERR_TIMEOUT, and the same context then partitions bit-exactly."""
    t0 = time.perf_counter()
    rc = ctx.lib.hp_test_wait_expiry(ctx.h)
    elapsed = time.perf_counter() - t0
    assert rc == HP_ERR_TIMEOUT
    assert elapsed < 60
    compare_runs(ctx, graphs.grid2d(40, 30, seed=6, wmin=1, wmax=5), 8)


def test_arena_exhaustion_retry(ctx):
    """The arena's grow-and-retry path, driven from the host: the first attempt
    gets a small arena, runs out, launches nothing more and restarts with twice
    the arena.  Four attempts that all run out return HP_ERR_NOMEM and leave
    the context usable; the first start size that succeeds does so after
    restarts, with the same partition as a call with the estimated arena."""
    g = graphs.rmat(14, seed=7)
    ref_part, ref_cut, _ = compare_runs(ctx, g, 16)
    lib, h = ctx.lib, ctx.h
    assert lib.hp_test_arena_first(h, -1) == HP_ERR_INVALID_ARG
    first = 64 << 10
    seen_nomem = False
    while True:
        assert lib.hp_test_arena_first(h, first) == 0
        try:
            part, cut = ctx.partition_graph(g, 16)
        except hp.HpError as e:
            assert e.code == HP_ERR_NOMEM
            assert lib.hp_test_arena_restarts(h) == 3
            seen_nomem = True
            first *= 2
            assert first <= 1 << 30
            continue
        break
    assert seen_nomem
    assert lib.hp_test_arena_restarts(h) >= 1
    assert np.array_equal(part, ref_part) and cut == ref_cut
    # an override cleared before use leaves the next call on the estimate
    assert lib.hp_test_arena_first(h, 1 << 20) == 0
    assert lib.hp_test_arena_first(h, 0) == 0
    part, cut = ctx.partition_graph(g, 16)
    assert lib.hp_test_arena_restarts(h) == 0
    assert np.array_equal(part, ref_part) and cut == ref_cut


def test_invalid_inputs(ctx):
    bad = np.array([0, 1, 2], np.int32)
    with pytest.raises(hp.HpError) as e:
        ctx.partition(bad, np.array([0, 0], np.int32), 2)         # self loop
    assert e.value.code == HP_ERR_INVALID_GRAPH
    with pytest.raises(hp.HpError) as e:
        ctx.partition(bad, np.array([5, 0], np.int32), 2)         # out of range
    assert e.value.code == HP_ERR_INVALID_GRAPH
    with pytest.raises(hp.HpError) as e:
        ctx.partition(bad, np.array([1, 0], np.int32), 2, adjwgt=np.array([0, 0], np.int32))
    assert e.value.code == HP_ERR_INVALID_GRAPH
    g = graphs.grid2d(4, 4)
    with pytest.raises(hp.HpError) as e:
        ctx.partition_graph(g, 0)
    assert e.value.code == HP_ERR_INVALID_ARG
    with pytest.raises(hp.HpError) as e:
        ctx.partition_graph(g, 20000)
    assert e.value.code == HP_ERR_UNSUPPORTED
    with pytest.raises(hp.HpError) as e:
        ctx.partition_graph(g, 4, ubfactor=0.9)
    assert e.value.code == HP_ERR_INVALID_ARG
    # the context stays usable after errors
    part, cut = ctx.partition_graph(g, 4)
    assert cut == oracle.edgecut(g, part)


def _csr(n, rows, weights=None):
    xadj = np.zeros(n + 1, np.int32)
    for v, r in enumerate(rows):
        xadj[v + 1] = xadj[v] + len(r)
    adj = np.array([u for r in rows for u in r], np.int32)
    w = None if weights is None else np.array([x for r in weights for x in r], np.int32)
    return xadj, adj, w


def test_invalid_asymmetric_and_duplicate(ctx):
    """Asymmetric adjacency (a missing reverse entry, or a weight that differs
    between the two directions) and duplicate neighbours (in a sorted row and
    in an unsorted one) are rejected with HP_ERR_INVALID_GRAPH; the reference's
    own checker is check_graph (hunyuangraph_GPU_match.h:1718-1800)."""
    # 0-1, 1-2, 2-3 path; vertex 3 lacks its entry for 2
    xadj, adj, _ = _csr(4, [[1], [0, 2], [1, 3], []])
    with pytest.raises(hp.HpError) as e:
        ctx.partition(xadj, adj, 2)
    assert e.value.code == HP_ERR_INVALID_GRAPH
    # symmetric structure, weight 5 one way and 6 the other
    xadj, adj, w = _csr(3, [[1], [0, 2], [1]], [[4], [4, 5], [6]])
    with pytest.raises(hp.HpError) as e:
        ctx.partition(xadj, adj, 2, adjwgt=w)
    assert e.value.code == HP_ERR_INVALID_GRAPH
    # duplicate neighbour in a sorted row (the pair 0-1 listed twice both ways)
    xadj, adj, _ = _csr(3, [[1, 1, 2], [0, 0], [0]])
    with pytest.raises(hp.HpError) as e:
        ctx.partition(xadj, adj, 2)
    assert e.value.code == HP_ERR_INVALID_GRAPH
    # the same in unsorted rows of a larger graph (the hash-table path)
    g = graphs.rmat(12, 8, seed=5)
    rows = [list(g.adjncy[g.xadj[v]:g.xadj[v + 1]][::-1]) for v in range(g.nvtxs)]
    v = int(np.argmax(np.diff(g.xadj)))
    u = rows[v][0]
    rows[v].append(u)
    rows[u].append(v)
    xadj, adj, _ = _csr(g.nvtxs, rows)
    with pytest.raises(hp.HpError) as e:
        ctx.partition(xadj, adj, 8)
    assert e.value.code == HP_ERR_INVALID_GRAPH
    # unsorted rows without duplicates are accepted and give the sorted graph's partition
    rows = [list(g.adjncy[g.xadj[v]:g.xadj[v + 1]][::-1]) for v in range(g.nvtxs)]
    xadj, adj, _ = _csr(g.nvtxs, rows)
    p_unsorted, c_unsorted = ctx.partition(xadj, adj, 8)
    assert c_unsorted == oracle.edgecut(graphs.Graph(xadj, adj, g.vwgt, np.ones_like(adj)), p_unsorted)
    # the context stays usable
    part, cut = ctx.partition_graph(graphs.grid2d(8, 8), 4)
    assert cut == oracle.edgecut(graphs.grid2d(8, 8), part)


def test_weight_range(ctx):
    """Edge weights whose sums could wrap the int32 coarse weights and
    connectivities: a vertex of any level with a weighted degree of 2^31 or
    more fails with HP_ERR_UNSUPPORTED, as in the oracle (on the input level,
    a star; on a coarse level, a heavy grid); a graph whose total weight
    exceeds 2^31 but whose vertices stay below it partitions exactly as the
    oracle does."""
    n = 9
    xadj = np.array([0, 8] + list(range(9, 17)), np.int32)
    adj = np.array(list(range(1, 9)) + [0] * 8, np.int32)
    star = graphs.Graph(xadj, adj, np.ones(n, np.int32), np.full(16, 1 << 29, np.int32))
    with pytest.raises(hp.HpError) as e:
        ctx.partition_graph(star, 2)
    assert e.value.code == HP_ERR_UNSUPPORTED
    g = graphs.grid2d(256, 256)
    heavy = graphs.Graph(g.xadj, g.adjncy, g.vwgt, np.full(g.nedges, 1 << 26, np.int32))
    with pytest.raises(hp.HpError) as e:
        ctx.partition_graph(heavy, 8)
    assert e.value.code == HP_ERR_UNSUPPORTED
    with pytest.raises(oracle.OracleError) as oe:
        oracle.partition(heavy, 8, 1.03)
    assert oe.value.code == HP_ERR_UNSUPPORTED
    # weight 2^21: total about 5.5e11, every vertex of every level below 2^31
    light = graphs.Graph(g.xadj, g.adjncy, g.vwgt, np.full(g.nedges, 1 << 21, np.int32))
    compare_runs(ctx, light, 8)
    part, cut = ctx.partition_graph(g, 4)
    assert cut == oracle.edgecut(g, part)

def test_legacy_entry_point(ctx):
    g = graphs.grid2d(40, 30, seed=3, wmin=1, wmax=9)
    lib = hp.load_library()
    I = C.POINTER(C.c_int32)
    p = lambda a: a.ctypes.data_as(I)  # noqa: E731
    n = C.c_int32(g.nvtxs)
    k = C.c_int32(6)
    ub = np.array([1.03], np.float32)
    part = np.full(g.nvtxs, -7, np.int32)
    lib.hunyuangraph_PartitionGraph(C.byref(n), p(g.xadj), p(g.adjncy), p(g.vwgt), p(g.adjwgt), C.byref(k),
                                    None, ub.ctypes.data_as(C.POINTER(C.c_float)), p(part))
    ref_part, _ = ctx.partition_graph(g, 6)
    assert np.array_equal(part, ref_part)
    # the Python mirror with the reference's argument list
    out = np.zeros(g.nvtxs, np.int32)
    hp.PartitionGraph(g.nvtxs, g.xadj, g.adjncy, g.vwgt, g.adjwgt, 6, None, [1.03], out)
    assert np.array_equal(out, ref_part)


def test_partition_device_torch(ctx):
    import torch
    g = graphs.grid3d(24, 24, 24, seed=2, wmin=1, wmax=10)
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(a).to(dev) for a in (g.xadj, g.adjncy, g.vwgt, g.adjwgt)]
    part, cut = ctx.partition_device(t[0], t[1], 32, t[2], t[3])
    torch.cuda.synchronize()
    ref_part, ref_cut = ctx.partition_graph(g, 32)
    assert cut == ref_cut
    assert np.array_equal(part.cpu().numpy(), ref_part)
    assert ctx.edgecut_device(t[0], t[1], t[3], part) == ref_cut


def hybrid_test_graph():
    """R-MAT scale 17 plus two hubs joined to 11,000 and 20,000 vertices with
    high ids: on level 0 (about 70K coarse ids) the long rows have entries on
    both sides of the hybrid contraction's dense range (ids below 32768), and
    the hubs' rows have more high ids than its 4096-entry buffer, so they spill
    to the CTA radix kernel (up to 12288 entries) and to the dense slab kernel
    (longer)."""
    g = graphs.rmat(17, 16, seed=11, wmin=1, wmax=100)
    n = g.nvtxs
    rng = np.random.default_rng(5)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(g.xadj))
    dst = g.adjncy.astype(np.int64)
    extra = []
    for hub, cnt in ((3, 11000), (5, 20000)):
        nb = rng.choice(np.arange(n // 2, n), size=cnt, replace=False)
        extra.append((np.full(cnt, hub), nb))
    es = np.concatenate([src] + [a for a, b in extra] + [b for a, b in extra])
    ed = np.concatenate([dst] + [b for a, b in extra] + [a for a, b in extra])
    key = np.unique(es * n + ed)                      # sorted, duplicates dropped
    s, d = key // n, key % n
    keep = s != d
    s, d = s[keep], d[keep]
    xadj = np.zeros(n + 1, np.int64)
    np.add.at(xadj, s + 1, 1)
    xadj = np.cumsum(xadj).astype(np.int32)
    lo, hi = np.minimum(s, d).astype(np.uint64), np.maximum(s, d).astype(np.uint64)
    w = ((lo * np.uint64(2654435761) + hi * np.uint64(40503)) % np.uint64(100) + np.uint64(1)).astype(np.int32)
    return graphs.Graph(xadj, d.astype(np.int32), np.ones(n, np.int32), w)


@pytest.mark.parametrize("hybrid", [1, 0])
def test_hybrid_contraction(ctx, hybrid):
    """The hybrid long-row contraction (dense shared-memory accumulation of the
    low coarse ids, radix sort of the rest, spills of rows whose rest does not
    fit) writes the same coarse rows as the radix path: every level equal to
    the oracle, with both settings, every level off the 48K shared-memory path."""
    g = hybrid_test_graph()
    ctx.set_tuning(contract_smem_cn=0, contract_hybrid=hybrid)
    try:
        compare_runs(ctx, g, 64)
    finally:
        ctx.set_tuning(None)
