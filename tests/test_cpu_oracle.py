"""CPU oracle: pinned against the reference's own CPU code (golden fixtures and,
when built, oracle/_ref) and checked for determinism and rule invariants."""
import ctypes as C
import glob
import json
import os

import numpy as np
import pytest

import oracle
from hunyuansc25_b200 import graphs
from hunyuansc25_b200._abi import default_options

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class G:
    def __init__(self, xadj, adjncy, vwgt, adjwgt):
        self.xadj, self.adjncy, self.vwgt, self.adjwgt = (np.ascontiguousarray(a, np.int32) for a in
                                                          (xadj, adjncy, vwgt, adjwgt))

    @property
    def nvtxs(self):
        return self.xadj.shape[0] - 1

    @property
    def nedges(self):
        return self.adjncy.shape[0]


def sorted_rows(xadj, adjncy, adjwgt):
    a = adjncy.copy()
    w = adjwgt.copy()
    for c in range(xadj.shape[0] - 1):
        s, e = xadj[c], xadj[c + 1]
        o = np.argsort(a[s:e], kind="stable")
        a[s:e] = a[s:e][o]
        w[s:e] = w[s:e][o]
    return a, w


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_contract_*.npz"))))
def test_contract_matches_reference_golden(path):
    d = np.load(path)
    g = G(d["xadj"], d["adjncy"], d["vwgt"], d["adjwgt"])
    cx, ca, cw, cv = oracle.contract(g, d["match"], d["cmap"], int(d["cn"]))
    assert np.array_equal(cx, d["cxadj"])
    assert np.array_equal(cv, d["cvwgt"])
    ra, rw = sorted_rows(d["cxadj"], d["cadjncy"], d["cadjwgt"])
    assert np.array_equal(ca, ra)
    assert np.array_equal(cw, rw)
    assert oracle.edgecut(g, d["part"]) == int(d["cut"])


def test_golden_fixtures_present():
    assert len(glob.glob(os.path.join(GOLDEN, "ref_contract_*.npz"))) >= 4
    assert len(glob.glob(os.path.join(GOLDEN, "ref_split_*.npz"))) >= 4


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_split_*.npz"))))
def test_split_matches_reference_golden(path):
    """The recursive bisection's split into induced subgraphs equals the
    reference's hunyuangraph_splitgraph on both sides, arrays and order."""
    d = np.load(path)
    g = G(d["xadj"], d["adjncy"], d["vwgt"], d["adjwgt"])
    for side in (0, 1):
        got = oracle.split(g, d["where"], side)
        for arr, name in zip(got, ("xadj", "adjncy", "adjwgt", "vwgt", "label")):
            assert np.array_equal(arr, d[f"s{side}_{name}"]), (side, name)


def test_split_rejects_non_binary_where():
    g = graphs.grid2d(4, 4)
    with pytest.raises(ValueError):
        oracle.split(g, np.full(g.nvtxs, 2, np.int32), 0)


@pytest.mark.skipif(not os.path.exists(oracle.REFLIB), reason="reference CPU harness not built")
def test_split_matches_reference_live():
    ref = C.CDLL(oracle.REFLIB)
    I = C.POINTER(C.c_int32)
    p = lambda a: a.ctypes.data_as(I)  # noqa: E731
    for gi, g in enumerate((graphs.grid3d(12, 11, 10, seed=8, wmin=1, wmax=10), graphs.rmat(11, 8, seed=21))):
        n, m = g.nvtxs, g.nedges
        for s in range(3):
            where = (np.random.default_rng(100 * gi + s).random(n) < 0.3 + 0.2 * s).astype(np.int32)
            for side in (0, 1):
                sn = C.c_int32()
                rx, rv, rl = (np.empty(n + 1, np.int32), np.empty(n, np.int32), np.empty(n, np.int32))
                ra, rw = np.empty(m, np.int32), np.empty(m, np.int32)
                mm = ref.ref_cpu_split(n, p(g.xadj), p(g.adjncy), p(g.vwgt), p(g.adjwgt), p(where), side,
                                       C.byref(sn), p(rx), p(ra), p(rw), p(rv), p(rl))
                k = sn.value
                ox, oa, ow, ov, ol = oracle.split(g, where, side)
                assert np.array_equal(ox, rx[:k + 1]) and np.array_equal(oa, ra[:mm])
                assert np.array_equal(ow, rw[:mm]) and np.array_equal(ov, rv[:k]) and np.array_equal(ol, rl[:k])


@pytest.mark.skipif(not os.path.exists(oracle.REFLIB), reason="reference CPU harness not built")
def test_contract_matches_reference_live():
    ref = C.CDLL(oracle.REFLIB)
    I = C.POINTER(C.c_int32)
    p = lambda a: a.ctypes.data_as(I)  # noqa: E731
    for g in (graphs.grid3d(14, 13, 12, seed=8, wmin=1, wmax=10), graphs.rmat(11, 8, seed=21)):
        m, cmap, cn = oracle.match(g, 0, 5, 1 << 30, 6)
        cx, ca, cw, cv = oracle.contract(g, m, cmap, cn)
        rx = np.empty(cn + 1, np.int32)
        ra = np.empty(g.nedges, np.int32)
        rw = np.empty(g.nedges, np.int32)
        rv = np.empty(cn, np.int32)
        mc = ref.ref_cpu_contract(g.nvtxs, p(g.xadj), p(g.adjncy), p(g.vwgt), p(g.adjwgt), p(m), p(cmap),
                                  cn, p(rx), p(ra), p(rw), p(rv))
        assert mc == ca.shape[0]
        assert np.array_equal(rx, cx) and np.array_equal(rv, cv)
        sa, sw = sorted_rows(rx, ra[:mc], rw[:mc])
        assert np.array_equal(sa, ca) and np.array_equal(sw, cw)
        part = (np.arange(g.nvtxs) % 5).astype(np.int32)
        assert ref.ref_cpu_edgecut(g.nvtxs, p(g.xadj), p(g.adjncy), p(g.adjwgt), p(part)) == \
            oracle.edgecut(g, part)


def digest(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()[:16]


def test_oracle_vcycle_snapshot():
    with open(os.path.join(GOLDEN, "oracle_vcycle.json")) as f:
        snap = json.load(f)
    cases = {"grid2d_256_k8": graphs.config_grid2d(),
             "grid3d_24_k16": graphs.grid3d(24, 24, 24, seed=2, wmin=1, wmax=10)}
    oracle.set_threads(2)
    for name, g in cases.items():
        s = snap[name]
        part, cut, tr = oracle.partition(g, s["k"], 1.03, opt=default_options(coarsen_to=s["coarsen_to"]),
                                         trace=True)
        assert cut == s["cut"]
        assert digest(part) == s["part"]
        assert tr.nlevels == len(s["levels"])
        for l, lv in enumerate(s["levels"]):
            n, m, cs, cf = tr.level(l)
            assert (n, m, cs, cf) == (lv["n"], lv["m"], lv["cut_start"], lv["cut_final"])
            assert digest(tr.array(l, 1)) == lv["adjncy"]
            assert digest(tr.array(l, 7)) == lv["where_final"]


def test_oracle_thread_invariance():
    g = graphs.rmat(12, 8, seed=3)
    res = []
    for th in (1, 3, 8):
        oracle.set_threads(th)
        part, cut, _ = oracle.partition(g, 16, 1.03, opt=default_options())
        res.append((cut, digest(part)))
    assert res[0] == res[1] == res[2]


def test_oracle_balance_and_cut():
    g = graphs.config_grid2d()
    oracle.set_threads(4)
    part, cut, _ = oracle.partition(g, 8, 1.03, opt=default_options(coarsen_to=160))
    pw = np.bincount(part, minlength=8)
    opt, mx = oracle.part_targets(g.nvtxs, 8, 1.03)
    assert pw.max() <= mx.max()
    assert cut == oracle.edgecut(g, part)
    assert cut < 1600   # 256x256 grid, 8 parts: a 2x4 block layout cuts 1024


def test_match_rule_invariants():
    g = graphs.grid3d(10, 10, 10, seed=2, wmin=1, wmax=10)
    n = g.nvtxs
    maxvwgt = 4
    m, cmap, cn = oracle.match(g, 0, 1, maxvwgt, 6)
    assert np.all(m[m] == np.arange(n))          # involution
    lead = np.arange(n) <= m
    assert cn == lead.sum()
    assert np.array_equal(cmap[lead], np.arange(cn))   # coarse ids by smaller endpoint
    assert np.array_equal(cmap, cmap[m])
    assert np.all(g.vwgt + g.vwgt[m] <= np.maximum(maxvwgt, 2 * g.vwgt))


def test_match_seed_changes_ties():
    g = graphs.config_grid2d()   # unit weights: only the seeded tie key decides
    m1, _, c1 = oracle.match(g, 0, 1, 1 << 30, 6)
    m2, _, c2 = oracle.match(g, 0, 2, 1 << 30, 6)
    assert not np.array_equal(m1, m2)
    assert c1 < 0.6 * g.nvtxs and c2 < 0.6 * g.nvtxs


def gain_bucket_np(gain, vwgt):
    g = np.float32(gain) / np.float32(max(vwgt, 1))
    if g > 0:
        return 0
    if g == 0:
        return 1
    t = 25
    g = np.float32(abs(g))
    if g < 1:
        while g < 1:
            g = np.float32(g * np.float32(1.5))
            t -= 1
        return max(t, 2)
    while g > 1:
        g = np.float32(g / np.float32(1.5))
        t += 1
    return min(t, 49)


def test_gain_bucket_float_semantics():
    rng = np.random.default_rng(0)
    for _ in range(3000):
        gain = int(rng.integers(-5000, 200))
        vw = int(rng.integers(1, 300))
        assert oracle.gain_bucket(gain, vw) == gain_bucket_np(gain, vw)


def test_part_targets():
    opt, mx = oracle.part_targets(65536, 8, 1.03)
    assert np.all(opt == 8192)
    assert np.all(mx == 8437)
    opt, mx = oracle.part_targets(1000, 3, 1.05, tpwgts=[0.5, 0.25, 0.25])
    assert list(opt) == [500, 250, 250]
    # ubfactor is a C float: 1.05f = 1.0499999523..., so 0.5 * 1000 * ub floors to 524
    assert list(mx) == [524, 262, 262]


def test_oracle_edge_cases():
    # empty graph, isolated vertices, k = 1, k > n
    g = graphs.grid2d(1, 1)
    part, cut, _ = oracle.partition(g, 4, 1.03)
    assert cut == 0 and part.shape == (1,)
    g = graphs.grid2d(5, 5)
    part, cut, _ = oracle.partition(g, 1, 1.03)
    assert cut == 0 and np.all(part == 0)
    part, cut, _ = oracle.partition(g, 40, 1.03)
    assert part.min() >= 0 and part.max() < 40
    assert cut == oracle.edgecut(g, part)


def test_weight_range_rule():
    """The weight-range rule shared with the library: when the total edge
    weight reaches 2^31, a vertex of any level whose weighted degree reaches
    2^31 fails the call (HP_ERR_UNSUPPORTED), since the int32 coarse weights
    and connectivities could wrap; below that the partition is the ordinary
    one."""
    from hunyuansc25_b200._abi import HP_ERR_UNSUPPORTED
    # a star: the centre's weighted degree is 8 * 2^29 = 2^32 on the input level
    n = 9
    xadj = np.array([0, 8] + list(range(9, 17)), np.int32)
    adj = np.array(list(range(1, 9)) + [0] * 8, np.int32)
    star = G(xadj, adj, np.ones(n, np.int32), np.full(16, 1 << 29, np.int32))
    assert not oracle.weight_range_ok(star)
    with pytest.raises(oracle.OracleError) as e:
        oracle.partition(star, 2, 1.03)
    assert e.value.code == HP_ERR_UNSUPPORTED
    # a 2-D grid of weight 2^26: the input fits (4 * 2^26), coarse vertices with
    # a perimeter of 32 fine edges or more do not
    g = graphs.grid2d(256, 256)
    heavy = G(g.xadj, g.adjncy, g.vwgt, np.full(g.nedges, 1 << 26, np.int32))
    assert oracle.weight_range_ok(heavy)
    with pytest.raises(oracle.OracleError) as e:
        oracle.partition(heavy, 8, 1.03)
    assert e.value.code == HP_ERR_UNSUPPORTED
    # weight 2^21: total about 5.5e11, every coarse vertex below 2^31
    light = G(g.xadj, g.adjncy, g.vwgt, np.full(g.nedges, 1 << 21, np.int32))
    part, cut, _ = oracle.partition(light, 8, 1.03)
    assert cut == oracle.edgecut(light, part)
