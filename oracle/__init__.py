"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a C restatement of the partition path (oracle/hp_oracle.c).  It is
imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
the product (hunyuansc25_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

from hunyuansc25_b200._abi import (HP_TRACE_ADJNCY, HP_TRACE_ADJWGT, HP_TRACE_CMAP,
                                   HP_TRACE_MATCH, HP_TRACE_VWGT, HP_TRACE_WHERE_FINAL,
                                   HP_TRACE_WHERE_START, HP_TRACE_XADJ, HpOptions,
                                   default_options)

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBPATH = os.path.join(HERE, "_build", "libhp_oracle.so")
REFLIB = os.path.join(HERE, "_ref", "libhp_ref.so")
_LIB = None

I32P = C.POINTER(C.c_int32)
I64P = C.POINTER(C.c_int64)


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "hp_oracle.c")
    deps = [src, os.path.join(HERE, "hp_oracle.h"), os.path.join(ROOT, "include", "hp_partition.h")]
    if (not force and os.path.exists(LIBPATH)
            and all(os.path.getmtime(d) <= os.path.getmtime(LIBPATH) for d in deps)):
        return LIBPATH
    os.makedirs(os.path.dirname(LIBPATH), exist_ok=True)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else (shutil.which("gcc") or "gcc")
    subprocess.check_call([cc, "-O2", "-fPIC", "-fopenmp", "-std=c11", "-Wall",
                           "-I", os.path.join(ROOT, "include"), "-shared", "-o", LIBPATH, src, "-lm"])
    return LIBPATH


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBPATH):
            build()
        L = C.CDLL(LIBPATH)
        L.ora_set_threads.argtypes = [C.c_int]
        L.ora_partition.argtypes = [C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, C.POINTER(C.c_float),
                                    C.c_float, C.POINTER(HpOptions), I32P, I64P, C.POINTER(C.c_void_p)]
        L.ora_partition.restype = C.c_int
        L.ora_weight_range_ok.argtypes = [C.c_int32, I32P, I32P]
        L.ora_weight_range_ok.restype = C.c_int
        L.ora_node_nd.argtypes = [C.c_int32, I32P, I32P, I32P, C.POINTER(HpOptions), I32P, I32P]
        L.ora_node_nd.restype = C.c_int
        L.ora_nd_separator.argtypes = [C.c_int32, I32P, I32P, I32P, I32P]
        L.ora_nd_separator.restype = None
        L.ora_cholesky_nnz.argtypes = [C.c_int32, I32P, I32P, I32P]
        L.ora_cholesky_nnz.restype = C.c_int64
        L.ora_trace_nlevels.argtypes = [C.c_void_p]
        L.ora_trace_level.argtypes = [C.c_void_p, C.c_int, I32P, I64P, I64P, I64P]
        L.ora_trace_copy.argtypes = [C.c_void_p, C.c_int, C.c_int, I32P, C.c_int64]
        L.ora_trace_free.argtypes = [C.c_void_p]
        L.ora_edgecut.argtypes = [C.c_int32, I32P, I32P, I32P, I32P]
        L.ora_edgecut.restype = C.c_int64
        L.ora_match.argtypes = [C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, C.c_uint64, C.c_int64,
                                C.c_int32, I32P, I32P]
        L.ora_match.restype = C.c_int32
        L.ora_contract.argtypes = [C.c_int32, I32P, I32P, I32P, I32P, I32P, I32P, C.c_int32,
                                   C.POINTER(I32P), C.POINTER(I32P), C.POINTER(I32P), C.POINTER(I32P)]
        L.ora_contract.restype = C.c_int64
        L.ora_split.argtypes = [C.c_int32, I32P, I32P, I32P, I32P, I32P, C.c_int32, I32P, I32P, I32P, I32P,
                                I32P, I32P]
        L.ora_split.restype = C.c_int64
        L.ora_free.argtypes = [C.c_void_p]
        L.ora_part_targets.argtypes = [C.c_int64, C.c_int32, C.POINTER(C.c_float), C.c_float, I64P, I64P]
        L.ora_bisect_ub_fx.argtypes = [C.c_float, C.c_int32]
        L.ora_bisect_ub_fx.restype = C.c_int64
        L.ora_initpart.argtypes = [C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, I64P, C.c_int64,
                                   C.c_int32, C.c_int32, I32P]
        L.ora_refine.argtypes = [C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, I64P, I64P, C.c_int32,
                                 C.c_int32, I32P, I32P]
        L.ora_refine.restype = C.c_int64
        F32 = C.POINTER(C.c_float)
        L.ora_mlp_forward.argtypes = [F32, F32, C.c_int64, F32]
        L.ora_mlp_loss_grad.argtypes = [F32, F32, F32, C.c_int64, F32]
        L.ora_mlp_loss_grad.restype = C.c_float
        L.ora_gain_bucket.argtypes = [C.c_int32, C.c_int32]
        L.ora_gain_bucket.restype = C.c_int32
        _LIB = L
    return _LIB


def _p(a, t=C.c_int32):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(t))


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def edgecut(g, where) -> int:
    where = i32(where)
    return int(lib().ora_edgecut(g.nvtxs, _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(where)))


class Trace:
    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if self.h:
            lib().ora_trace_free(self.h)
            self.h = None

    @property
    def nlevels(self) -> int:
        return int(lib().ora_trace_nlevels(self.h))

    def level(self, l):
        n = C.c_int32()
        m = C.c_int64()
        cs = C.c_int64()
        cf = C.c_int64()
        rc = lib().ora_trace_level(self.h, l, C.byref(n), C.byref(m), C.byref(cs), C.byref(cf))
        assert rc == 0
        return n.value, m.value, cs.value, cf.value

    def array(self, l, what):
        n, m, _, _ = self.level(l)
        size = {HP_TRACE_XADJ: n + 1, HP_TRACE_ADJNCY: m, HP_TRACE_ADJWGT: m}.get(what, n)
        out = np.empty(max(size, 1), dtype=np.int32)
        rc = lib().ora_trace_copy(self.h, l, what, _p(out), out.shape[0])
        if rc != 0:
            return None
        return out[:size]


class OracleError(RuntimeError):
    """A non-zero return of ora_partition; .code is the HP_ERR_* value."""

    def __init__(self, code: int):
        self.code = code
        super().__init__(f"ora_partition failed: {code}")


def partition(g, nparts, ubfactor=1.03, tpwgts=None, opt: HpOptions | None = None, trace=False):
    """Full oracle V-cycle. Returns (part, cut, Trace|None)."""
    if opt is None:
        opt = default_options()
    part = np.empty(max(g.nvtxs, 1), dtype=np.int32)
    cut = C.c_int64()
    th = C.c_void_p()
    tp = None
    if tpwgts is not None:
        tp = np.ascontiguousarray(tpwgts, dtype=np.float32)
    rc = lib().ora_partition(g.nvtxs, _p(i32(g.xadj)), _p(i32(g.adjncy)), _p(i32(g.vwgt)),
                             _p(i32(g.adjwgt)), nparts, _p(tp, C.c_float) if tp is not None else None,
                             C.c_float(ubfactor), C.byref(opt), _p(part), C.byref(cut),
                             C.byref(th) if trace else None)
    if rc != 0:
        raise OracleError(rc)
    return part[:g.nvtxs], cut.value, (Trace(th.value) if trace else None)


def node_nd(g, opt: HpOptions | None = None):
    """Nested-dissection ordering (the library's hp_node_nd rules):
    (perm, iperm) with perm[new] = old and iperm[old] = new."""
    n = g.nvtxs
    perm = np.empty(max(n, 1), np.int32)
    iperm = np.empty(max(n, 1), np.int32)
    rc = lib().ora_node_nd(n, _p(i32(g.xadj)), _p(i32(g.adjncy)), _p(i32(g.vwgt)),
                           C.byref(opt if opt is not None else default_options()), _p(perm), _p(iperm))
    if rc != 0:
        raise OracleError(rc)
    return perm[:n], iperm[:n]


def nd_separator(g, where):
    """side_of in {0, 1, 2 = separator} from a 2-way partition (ND's rule)."""
    out = np.empty(max(g.nvtxs, 1), np.int32)
    lib().ora_nd_separator(g.nvtxs, _p(i32(g.xadj)), _p(i32(g.adjncy)), _p(i32(where)), _p(out))
    return out[:g.nvtxs]


def cholesky_nnz(g, iperm) -> int:
    """Entries of the Cholesky factor (diagonal included) under iperm."""
    return int(lib().ora_cholesky_nnz(g.nvtxs, _p(i32(g.xadj)), _p(i32(g.adjncy)), _p(i32(iperm))))


def weight_range_ok(g) -> bool:
    """The weight-range rule: every vertex's weighted degree is below 2^31."""
    return bool(lib().ora_weight_range_ok(g.nvtxs, _p(i32(g.xadj)), _p(i32(g.adjwgt))))


def match(g, level, seed, maxvwgt, rounds):
    n = g.nvtxs
    m_ = np.empty(max(n, 1), np.int32)
    cm = np.empty(max(n, 1), np.int32)
    cn = lib().ora_match(n, _p(g.xadj), _p(g.adjncy), _p(g.vwgt), _p(g.adjwgt), level, seed,
                         maxvwgt, rounds, _p(m_), _p(cm))
    return m_[:n], cm[:n], int(cn)


def contract(g, match_, cmap, cn):
    px, pa, pw, pv = I32P(), I32P(), I32P(), I32P()
    m = lib().ora_contract(g.nvtxs, _p(g.xadj), _p(g.adjncy), _p(g.vwgt), _p(g.adjwgt),
                           _p(i32(match_)), _p(i32(cmap)), cn, C.byref(px), C.byref(pa),
                           C.byref(pw), C.byref(pv))
    out = (np.ctypeslib.as_array(px, shape=(cn + 1,)).copy(),
           np.ctypeslib.as_array(pa, shape=(max(m, 1),))[:m].copy(),
           np.ctypeslib.as_array(pw, shape=(max(m, 1),))[:m].copy(),
           np.ctypeslib.as_array(pv, shape=(max(cn, 1),))[:cn].copy())
    for p in (px, pa, pw, pv):
        lib().ora_free(C.cast(p, C.c_void_p))
    return out


def split(g, where, side):
    """One side of the 2-way split the recursive bisection makes:
    (xadj, adjncy, adjwgt, vwgt, label) of the induced subgraph."""
    n, m = g.nvtxs, g.nedges
    sn = C.c_int32()
    sx = np.empty(n + 1, np.int32)
    sa = np.empty(max(m, 1), np.int32)
    sw = np.empty(max(m, 1), np.int32)
    sv = np.empty(max(n, 1), np.int32)
    sl = np.empty(max(n, 1), np.int32)
    mm = lib().ora_split(n, _p(i32(g.xadj)), _p(i32(g.adjncy)), _p(i32(g.vwgt)), _p(i32(g.adjwgt)),
                         _p(i32(where)), side, C.byref(sn), _p(sx), _p(sa), _p(sw), _p(sv), _p(sl))
    if mm < 0:
        raise ValueError("where[] must hold 0 or 1")
    k = sn.value
    return sx[:k + 1], sa[:mm], sw[:mm], sv[:k], sl[:k]


def part_targets(tvwgt, nparts, ubfactor, tpwgts=None):
    opt = np.empty(nparts, np.int64)
    mx = np.empty(nparts, np.int64)
    tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, np.float32)
    lib().ora_part_targets(tvwgt, nparts, _p(tp, C.c_float) if tp is not None else None,
                           C.c_float(ubfactor), _p(opt, C.c_int64), _p(mx, C.c_int64))
    return opt, mx


def gain_bucket(gain, vwgt):
    return int(lib().ora_gain_bucket(gain, vwgt))


def mlp_forward(params, x):
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty(x.shape[0], np.float32)
    F32 = C.POINTER(C.c_float)
    lib().ora_mlp_forward(params.ctypes.data_as(F32), x.ctypes.data_as(F32), x.shape[0], out.ctypes.data_as(F32))
    return out


def mlp_loss_grad(params, x, y):
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    g = np.empty(params.shape[0], np.float32)
    F32 = C.POINTER(C.c_float)
    loss = lib().ora_mlp_loss_grad(params.ctypes.data_as(F32), x.ctypes.data_as(F32), y.ctypes.data_as(F32),
                                   x.shape[0], g.ctypes.data_as(F32))
    return float(loss), g
