"""Generate the golden fixtures in tests/golden/ (run once, commit the outputs).

* ref_contract_*.npz — the reference's own CPU contraction
  (hunyuangraph_cpu_create_cgraph, hunyuangraph_CPU_contraction.h:9-100) and CPU
  edge cut (hunyuangraph_computecut_cpu, hunyuangraph_graph.h:144-155), run
  through oracle/_ref/libhp_ref.so (built from the reference sources by
  oracle/build_ref.sh), on small seeded graphs with a seeded matching.
* ref_split_*.npz — the reference's own CPU graph split (hunyuangraph_splitgraph,
  hunyuangraph_CPU_splitgraph.h:8-167), both sides, on the same graphs with a
  seeded 2-way partition.
* oracle_vcycle.json — per-level sizes, cuts and array digests of the oracle's
  V-cycle on the 256x256 grid workload (k = 8) and a 3-D grid, so that any
  change of the oracle's rules is visible in review.

Usage: python tests/golden/make_golden.py
"""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hunyuansc25_b200 import graphs  # noqa: E402
from hunyuansc25_b200._abi import default_options  # noqa: E402
import oracle  # noqa: E402

I = C.POINTER(C.c_int32)


def p(a):
    return a.ctypes.data_as(I)


def seeded_matching(g, seed):
    """A valid matching built from a seeded random order (independent of the
    oracle's rule): visit vertices in a random order, pair with the first
    unmatched neighbour."""
    rng = np.random.default_rng(seed)
    n = g.nvtxs
    match = -np.ones(n, np.int32)
    for v in rng.permutation(n):
        if match[v] != -1:
            continue
        for u in g.adjncy[g.xadj[v]:g.xadj[v + 1]]:
            if match[u] == -1 and u != v:
                match[v] = u
                match[u] = v
                break
    cmap = np.empty(n, np.int32)
    cn = 0
    for v in range(n):
        if match[v] == -1:
            match[v] = v
        if v <= match[v]:
            cmap[v] = cn
            cn += 1
    for v in range(n):
        if v > match[v]:
            cmap[v] = cmap[match[v]]
    return match, cmap, cn


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()[:16]


def cases():
    return {
        "grid2d_16x16_w": graphs.grid2d(16, 16, seed=9, wmin=1, wmax=20),
        "grid3d_6": graphs.grid3d(6, 6, 6, seed=2, wmin=1, wmax=10),
        "rmat_s8": graphs.rmat(8, 8, seed=3, wmin=1, wmax=100),
        "rgg_600": graphs.rgg(600, 10.0, seed=4),
    }


def make_split_fixtures(ref):
    """Both sides of the reference's split under a seeded 2-way partition."""
    for name, g in cases().items():
        n, m = g.nvtxs, g.nedges
        where = (np.random.default_rng(77).random(n) < 0.4).astype(np.int32)
        out = {"xadj": g.xadj, "adjncy": g.adjncy, "vwgt": g.vwgt, "adjwgt": g.adjwgt, "where": where}
        for side in (0, 1):
            sn = C.c_int32()
            sx = np.empty(n + 1, np.int32)
            sa = np.empty(max(m, 1), np.int32)
            sw = np.empty(max(m, 1), np.int32)
            sv = np.empty(max(n, 1), np.int32)
            sl = np.empty(max(n, 1), np.int32)
            mm = ref.ref_cpu_split(n, p(g.xadj), p(g.adjncy), p(g.vwgt), p(g.adjwgt), p(where), side,
                                   C.byref(sn), p(sx), p(sa), p(sw), p(sv), p(sl))
            k = sn.value
            out.update({f"s{side}_xadj": sx[:k + 1], f"s{side}_adjncy": sa[:mm], f"s{side}_adjwgt": sw[:mm],
                        f"s{side}_vwgt": sv[:k], f"s{side}_label": sl[:k]})
            print(name, "side", side, k, mm)
        np.savez_compressed(os.path.join(HERE, f"ref_split_{name}.npz"), **out)


def main():
    ref = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libhp_ref.so"))
    for name, g in cases().items():
        match, cmap, cn = seeded_matching(g, 1234)
        rx = np.empty(cn + 1, np.int32)
        ra = np.empty(g.nedges, np.int32)
        rw = np.empty(g.nedges, np.int32)
        rv = np.empty(cn, np.int32)
        mc = ref.ref_cpu_contract(g.nvtxs, p(g.xadj), p(g.adjncy), p(g.vwgt), p(g.adjwgt), p(match),
                                  p(cmap), cn, p(rx), p(ra), p(rw), p(rv))
        part = ((np.arange(g.nvtxs, dtype=np.int64) * 2654435761) % 7).astype(np.int32)
        cut = ref.ref_cpu_edgecut(g.nvtxs, p(g.xadj), p(g.adjncy), p(g.adjwgt), p(part))
        np.savez_compressed(os.path.join(HERE, f"ref_contract_{name}.npz"),
                            xadj=g.xadj, adjncy=g.adjncy, vwgt=g.vwgt, adjwgt=g.adjwgt,
                            match=match, cmap=cmap, cn=np.int32(cn), cxadj=rx, cadjncy=ra[:mc],
                            cadjwgt=rw[:mc], cvwgt=rv, part=part, cut=np.int64(cut))
        print(name, g.nvtxs, g.nedges, "->", cn, mc, "cut", cut)
    make_split_fixtures(ref)

    oracle.set_threads(4)
    snap = {}
    for name, g, k, ct in (("grid2d_256_k8", graphs.config_grid2d(), 8, 160),
                           ("grid3d_24_k16", graphs.grid3d(24, 24, 24, seed=2, wmin=1, wmax=10), 16, 0)):
        opt = default_options(coarsen_to=ct)
        part, cut, tr = oracle.partition(g, k, 1.03, opt=opt, trace=True)
        levels = []
        for l in range(tr.nlevels):
            n, m, cs, cf = tr.level(l)
            levels.append({"n": n, "m": m, "cut_start": cs, "cut_final": cf,
                           "adjncy": digest(tr.array(l, 1)), "where_final": digest(tr.array(l, 7))})
        snap[name] = {"k": k, "coarsen_to": ct, "cut": cut, "part": digest(part), "levels": levels}
        print(name, "cut", cut, "levels", tr.nlevels)
    with open(os.path.join(HERE, "oracle_vcycle.json"), "w") as f:
        json.dump(snap, f, indent=1)


if __name__ == "__main__":
    main()
