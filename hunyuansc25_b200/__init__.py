"""hunyuansc25_b200 — B200-native multilevel k-way graph partitioner.

Python mirror of the reference's partition entry point
(``hunyuangraph_PartitionGraph``, hunyuangraph_partitiongraph.h:284-347) over the
C ABI in ``include/hp_partition.h``.  Everything runs in the CUDA library
``lib/libhp_b200.so`` (sm_100a); there is no CPU fallback: if the library or a
CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._abi import (ERROR_NAMES, HP_MLP_NPARAM, HP_OK, HP_TRACE_ADJNCY, HP_TRACE_ADJWGT, HP_TRACE_CMAP,
                   HP_TRACE_MATCH, HP_TRACE_VWGT, HP_TRACE_WHERE_FINAL, HP_TRACE_WHERE_START,
                   HP_TRACE_XADJ, PROTOTYPES, HpOptions, HpStats, HpTuning, default_options)

__all__ = [
    "HpError", "Context", "partition_graph", "PartitionGraph", "default_options", "HpOptions",
    "HpStats", "library_path", "load_library",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def library_path() -> str:
    return os.path.join(_HERE, "lib", "libhp_b200.so")


class HpError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        name = ERROR_NAMES.get(code, str(code))
        msg = f"{what}: {name}" if what else name
        lib = _LIB
        if lib is not None:
            try:
                msg += f" ({lib.hp_strerror(code).decode()})"
            except Exception:  # pragma: no cover
                pass
        super().__init__(msg)


def load_library():
    """Load the CUDA library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} is missing: build it with `python -m hunyuansc25_b200.build`")
        lib = C.CDLL(path)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _check(rc, what):
    if rc != HP_OK:
        raise HpError(rc, what)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p32(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


class BatchInput:
    """Concatenated host arrays of many graphs in hp_partition_batch's layout
    (Context.prepare_batch), with the output buffers."""


class Context:
    """One device arena + per-call state (reentrant replacement of the
    reference's file-scope globals, hunyuangraph_GPU_memory.h:18-32)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.hp_context_create(device, C.byref(h)), "hp_context_create")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.hp_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- partition ----------------------------------------------------------------
    def partition(self, xadj, adjncy, nparts, vwgt=None, adjwgt=None, ubfactor=1.03,
                  tpwgts=None, options: HpOptions | None = None):
        """Host arrays in, (part, edgecut) out."""
        xadj = _i32(xadj)
        adjncy = _i32(adjncy)
        vwgt = None if vwgt is None else _i32(vwgt)
        adjwgt = None if adjwgt is None else _i32(adjwgt)
        n = xadj.shape[0] - 1
        part = np.empty(max(n, 1), dtype=np.int32)
        cut = C.c_int64()
        tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
        opt = options if options is not None else default_options()
        rc = self.lib.hp_partition(self.h, n, _p32(xadj), _p32(adjncy), _p32(vwgt), _p32(adjwgt),
                                   nparts, None if tp is None else tp.ctypes.data_as(C.POINTER(C.c_float)),
                                   C.c_float(ubfactor), C.byref(opt), _p32(part), C.byref(cut))
        _check(rc, "hp_partition")
        return part[:n], cut.value

    def partition_graph(self, g, nparts, ubfactor=1.03, tpwgts=None, options=None):
        return self.partition(g.xadj, g.adjncy, nparts, g.vwgt, g.adjwgt, ubfactor, tpwgts, options)

    def partition_device(self, xadj, adjncy, nparts, vwgt=None, adjwgt=None, ubfactor=1.03,
                         tpwgts=None, options: HpOptions | None = None, stream=None, part=None):
        """torch CUDA int32 tensors in (device-resident), (part tensor, cut) out."""
        import torch
        n = xadj.numel() - 1
        if part is None:
            part = torch.empty(max(n, 1), dtype=torch.int32, device=xadj.device)
        cut = C.c_int64()
        tp = None if tpwgts is None else np.ascontiguousarray(tpwgts, dtype=np.float32)
        opt = options if options is not None else default_options()
        s = stream if stream is not None else torch.cuda.current_stream(xadj.device)
        rc = self.lib.hp_partition_device(
            self.h, n, adjncy.numel(), C.c_void_p(xadj.data_ptr()), C.c_void_p(adjncy.data_ptr()),
            C.c_void_p(vwgt.data_ptr()) if vwgt is not None else None,
            C.c_void_p(adjwgt.data_ptr()) if adjwgt is not None else None, nparts,
            None if tp is None else tp.ctypes.data_as(C.POINTER(C.c_float)), C.c_float(ubfactor),
            C.byref(opt), C.c_void_p(s.cuda_stream), C.c_void_p(part.data_ptr()), C.byref(cut))
        _check(rc, "hp_partition_device")
        return part[:n], cut.value

    def prepare_batch(self, graphs, nparts, ubfactor=1.03) -> "BatchInput":
        """The concatenated host arrays of hp_partition_batch for these graphs
        (built once; partition_prepared() can run them many times)."""
        G = len(graphs)
        b = BatchInput()
        b.G = G
        b.nparts = np.ascontiguousarray(np.broadcast_to(np.asarray(nparts, np.int32), (G,)))
        b.ub = np.ascontiguousarray(np.broadcast_to(np.asarray(ubfactor, np.float32), (G,)))
        b.vtx = np.zeros(G + 1, np.int64)
        b.edg = np.zeros(G + 1, np.int64)
        for i, g in enumerate(graphs):
            b.vtx[i + 1] = b.vtx[i] + g.nvtxs
            b.edg[i + 1] = b.edg[i] + g.nedges
        b.xadj = np.concatenate([g.xadj for g in graphs]).astype(np.int32)
        b.adj = np.concatenate([g.adjncy for g in graphs]).astype(np.int32)
        b.vw = np.concatenate([g.vwgt for g in graphs]).astype(np.int32)
        b.ew = np.concatenate([g.adjwgt for g in graphs]).astype(np.int32)
        b.part = np.empty(max(int(b.vtx[-1]), 1), np.int32)
        b.cuts = np.zeros(G, np.int64)
        return b

    def partition_prepared(self, b: "BatchInput", options=None):
        """One hp_partition_batch call on prepared arrays; returns (list of part
        arrays, cuts) -- views of the BatchInput's output arrays."""
        opt = options if options is not None else default_options()
        I64 = C.POINTER(C.c_int64)
        rc = self.lib.hp_partition_batch(self.h, b.G, b.vtx.ctypes.data_as(I64), b.edg.ctypes.data_as(I64),
                                         _p32(b.xadj), _p32(b.adj), _p32(b.vw), _p32(b.ew), _p32(b.nparts),
                                         b.ub.ctypes.data_as(C.POINTER(C.c_float)), C.byref(opt),
                                         _p32(b.part), b.cuts.ctypes.data_as(I64))
        _check(rc, "hp_partition_batch")
        return [b.part[b.vtx[i]:b.vtx[i + 1]] for i in range(b.G)], b.cuts

    def partition_batch(self, graphs, nparts, ubfactor=1.03, options=None):
        """Partition many independent graphs; returns (list of part arrays, cuts)."""
        b = self.prepare_batch(graphs, nparts, ubfactor)
        parts, cuts = self.partition_prepared(b, options)
        return [p.copy() for p in parts], cuts.copy()

    def stats(self) -> HpStats:
        st = HpStats()
        _check(self.lib.hp_last_stats(self.h, C.byref(st)), "hp_last_stats")
        return st

    # ---- nested-dissection ordering ---------------------------------------------------
    def node_nd(self, xadj, adjncy, vwgt=None, options: HpOptions | None = None):
        """Fill-reducing nested-dissection ordering of a host CSR (hp_node_nd):
        (perm, iperm) with perm[new] = old and iperm[old] = new."""
        xadj = _i32(xadj)
        adjncy = _i32(adjncy)
        vwgt = None if vwgt is None else _i32(vwgt)
        n = xadj.shape[0] - 1
        perm = np.empty(max(n, 1), np.int32)
        iperm = np.empty(max(n, 1), np.int32)
        opt = options if options is not None else default_options()
        _check(self.lib.hp_node_nd(self.h, n, _p32(xadj), _p32(adjncy), _p32(vwgt), C.byref(opt), _p32(perm),
                                   _p32(iperm)), "hp_node_nd")
        return perm[:n], iperm[:n]

    def node_nd_graph(self, g, options=None):
        return self.node_nd(g.xadj, g.adjncy, g.vwgt, options)

    # ---- trace ----------------------------------------------------------------------
    @property
    def trace_nlevels(self) -> int:
        return int(self.lib.hp_trace_nlevels(self.h))

    def trace_level(self, level):
        n = C.c_int32()
        m = C.c_int64()
        cs = C.c_int64()
        cf = C.c_int64()
        _check(self.lib.hp_trace_level(self.h, level, C.byref(n), C.byref(m), C.byref(cs),
                                       C.byref(cf)), "hp_trace_level")
        return n.value, m.value, cs.value, cf.value

    def trace_array(self, level, what):
        n, m, _, _ = self.trace_level(level)
        size = {HP_TRACE_XADJ: n + 1, HP_TRACE_ADJNCY: m, HP_TRACE_ADJWGT: m}.get(what, n)
        out = np.empty(max(size, 1), dtype=np.int32)
        rc = self.lib.hp_trace_copy(self.h, level, what, _p32(out), out.shape[0])
        if rc != HP_OK:
            return None
        return out[:size]

    # ---- kernel tuning ---------------------------------------------------------------
    def set_tuning(self, tuning=None, **fields):
        """Installs a kernel tuning (speed only; the partition does not change).
        ``tuning`` is a dict of hp_tuning fields (missing ones take their
        defaults) or None for the defaults; keyword fields override it."""
        d = dict(tuning or {})
        d.update(fields)
        t = HpTuning.from_dict(d)
        _check(self.lib.hp_context_set_tuning(self.h, C.byref(t)), "hp_context_set_tuning")

    def get_tuning(self) -> dict:
        t = HpTuning()
        _check(self.lib.hp_context_get_tuning(self.h, C.byref(t)), "hp_context_get_tuning")
        return t.as_dict()

    def load_tuning(self, path: str) -> dict:
        """Installs the tuning stored in a tuning file (hunyuansc25_b200.tune)."""
        from . import tune
        t = tune.read_tuning_file(path)
        self.set_tuning(t)
        return t

    # ---- learned move proposals -------------------------------------------------------
    def mlp_set_params(self, params, threshold: float = 0.0):
        params = np.ascontiguousarray(params, dtype=np.float32)
        _check(self.lib.hp_mlp_set_params(self.h, params.ctypes.data_as(C.POINTER(C.c_float)), params.shape[0],
                                          C.c_float(threshold)), "hp_mlp_set_params")

    def mlp_get_params(self):
        out = np.empty(HP_MLP_NPARAM, np.float32)
        _check(self.lib.hp_mlp_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), HP_MLP_NPARAM),
               "hp_mlp_get_params")
        return out

    def mlp_loss_grad(self, x, y):
        """x: CUDA float32 [n, 8], y: CUDA float32 [n] -> (loss, grad numpy)."""
        g = np.empty(HP_MLP_NPARAM, np.float32)
        loss = C.c_float()
        _check(self.lib.hp_mlp_loss_grad(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), y.numel(),
                                         g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)),
               "hp_mlp_loss_grad")
        return loss.value, g

    def mlp_train(self, x, y, perm=None, epochs=1, batch=4096, lr=3e-3):
        loss = C.c_float()
        _check(self.lib.hp_mlp_train(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                     C.c_void_p(perm.data_ptr()) if perm is not None else None, y.numel(),
                                     epochs, batch, C.c_float(lr), C.byref(loss)), "hp_mlp_train")
        return loss.value

    def mlp_infer(self, x, tensor_cores=True):
        import torch
        out = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        _check(self.lib.hp_mlp_infer(self.h, C.c_void_p(x.data_ptr()), x.shape[0], C.c_void_p(out.data_ptr()),
                                     1 if tensor_cores else 0), "hp_mlp_infer")
        return out

    def movelog_enable(self, capacity: int):
        _check(self.lib.hp_movelog_enable(self.h, capacity), "hp_movelog_enable")

    def movelog_count(self) -> int:
        return int(self.lib.hp_movelog_count(self.h))

    def movelog_fetch(self):
        n = self.movelog_count()
        x = np.empty((max(n, 1), 8), np.float32)
        y = np.empty(max(n, 1), np.float32)
        _check(self.lib.hp_movelog_copy(self.h, x.ctypes.data_as(C.POINTER(C.c_float)),
                                        y.ctypes.data_as(C.POINTER(C.c_float)), n), "hp_movelog_copy")
        return x[:n], y[:n]

    def movelog_reset(self):
        _check(self.lib.hp_movelog_reset(self.h), "hp_movelog_reset")

    # ---- primitives -------------------------------------------------------------------
    def scan_exclusive(self, d_in, d_out=None, stream=None):
        """Exclusive int32 scan of a CUDA tensor; returns a tensor of n+1 entries."""
        import torch
        n = d_in.numel()
        if d_out is None:
            d_out = torch.empty(n + 1, dtype=torch.int32, device=d_in.device)
        s = stream if stream is not None else torch.cuda.current_stream(d_in.device)
        _check(self.lib.hp_scan_exclusive_i32(self.h, C.c_void_p(d_in.data_ptr()),
                                              C.c_void_p(d_out.data_ptr()), n,
                                              C.c_void_p(s.cuda_stream)), "hp_scan_exclusive_i32")
        return d_out

    def edgecut_device(self, xadj, adjncy, adjwgt, where, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream(xadj.device)
        cut = C.c_int64()
        _check(self.lib.hp_edgecut_device(self.h, xadj.numel() - 1, C.c_void_p(xadj.data_ptr()),
                                          C.c_void_p(adjncy.data_ptr()),
                                          C.c_void_p(adjwgt.data_ptr()) if adjwgt is not None else None,
                                          C.c_void_p(where.data_ptr()), C.c_void_p(s.cuda_stream),
                                          C.byref(cut)), "hp_edgecut_device")
        return cut.value


_DEFAULT_CTX = None


def _default_ctx() -> Context:
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


def partition_graph(xadj, adjncy, nparts, vwgt=None, adjwgt=None, ubfactor=1.03, tpwgts=None,
                    options=None):
    """Functional form of ``hunyuangraph_PartitionGraph``: returns (part, edgecut)."""
    return _default_ctx().partition(xadj, adjncy, nparts, vwgt, adjwgt, ubfactor, tpwgts, options)


def PartitionGraph(nvtxs, xadj, adjncy, vwgt, adjwgt, nparts, tpwgts, ubvec, part):
    """Argument-for-argument mirror of the reference's
    ``hunyuangraph_PartitionGraph(nvtxs, xadj, adjncy, vwgt, adjwgt, nparts, tpwgts,
    ubvec, part)`` (hunyuangraph_partitiongraph.h:284): writes into ``part``."""
    ub = float(ubvec[0]) if ubvec is not None else 1.03
    p, _ = partition_graph(np.asarray(xadj)[: nvtxs + 1], adjncy, nparts, vwgt, adjwgt, ub, tpwgts)
    part[:nvtxs] = p
