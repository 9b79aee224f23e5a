"""Seeded synthetic graphs (numpy CSR) built by the native generators (include/hp_gen.h).

The partition workloads, with the shapes the reference's benchmark graphs stand for:

* ``grid2d``  — 2-D 5-point grid (256 x 256, unit weights, k = 8)
* ``grid3d``  — 3-D 7-point grid (128^3, edge weights U{1..10}, k = 64)
* ``rmat``    — R-MAT scale 22, edge factor 16, a/b/c/d = .57/.19/.19/.05,
  edge weights U{1..100}, k = 256
* ``rgg``     — random geometric graph, 2^24 points, mean degree 12,
  w = int(1000 (1 - d/r)) + 1, k = 1024
* ``batch``   — 1,024 graphs, n log-uniform in [1e3, 2e5], half grids, half R-MAT
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class _HpGraph(C.Structure):
    _fields_ = [
        ("nvtxs", C.c_int32),
        ("nedges", C.c_int64),
        ("xadj", C.POINTER(C.c_int32)),
        ("adjncy", C.POINTER(C.c_int32)),
        ("vwgt", C.POINTER(C.c_int32)),
        ("adjwgt", C.POINTER(C.c_int32)),
    ]


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "lib", "libhp_gen.so")
        if not os.path.exists(path):
            from . import build
            build.build_gen()
        lib = C.CDLL(path)
        lib.hp_gen_grid2d.argtypes = [C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int32,
                                      C.POINTER(_HpGraph)]
        lib.hp_gen_grid3d.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                                      C.c_int32, C.POINTER(_HpGraph)]
        lib.hp_gen_rmat.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                    C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                    C.POINTER(_HpGraph)]
        lib.hp_gen_rgg.argtypes = [C.c_int32, C.c_double, C.c_uint64, C.POINTER(_HpGraph)]
        lib.hp_graph_free.argtypes = [C.POINTER(_HpGraph)]
        lib.hp_gen_set_threads.argtypes = [C.c_int]
        lib.hp_gen_edge_weight.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        lib.hp_gen_edge_weight.restype = C.c_int32
        lib.hp_read_metis.argtypes = [C.c_char_p, C.POINTER(_HpGraph), C.c_char_p, C.c_int]
        lib.hp_write_partition.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.c_int32, C.c_int32]
        lib.hp_write_metis.argtypes = [C.c_char_p, C.POINTER(_HpGraph)]
        lib.hp_read_mtx.argtypes = [C.c_char_p, C.POINTER(_HpGraph), C.c_char_p, C.c_int]
        _LIB = lib
    return _LIB


@dataclass
class Graph:
    """CSR graph: int32 arrays, symmetric, rows sorted."""

    xadj: np.ndarray
    adjncy: np.ndarray
    vwgt: np.ndarray
    adjwgt: np.ndarray
    name: str = ""

    @property
    def nvtxs(self) -> int:
        return int(self.xadj.shape[0] - 1)

    @property
    def nedges(self) -> int:
        """Directed adjacency entries (2 x undirected edges)."""
        return int(self.adjncy.shape[0])

    @property
    def nbytes(self) -> int:
        return sum(a.nbytes for a in (self.xadj, self.adjncy, self.vwgt, self.adjwgt))


def _take(g: _HpGraph, name: str) -> Graph:
    n, m = int(g.nvtxs), int(g.nedges)
    out = Graph(
        xadj=np.ctypeslib.as_array(g.xadj, shape=(n + 1,)).copy(),
        adjncy=np.ctypeslib.as_array(g.adjncy, shape=(max(m, 1),))[:m].copy(),
        vwgt=np.ctypeslib.as_array(g.vwgt, shape=(max(n, 1),))[:n].copy(),
        adjwgt=np.ctypeslib.as_array(g.adjwgt, shape=(max(m, 1),))[:m].copy(),
        name=name,
    )
    _lib().hp_graph_free(C.byref(g))
    return out


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with code {rc}")


def read_metis(path: str) -> Graph:
    """Read a METIS .graph file (replaces hunyuangraph_readgraph, hunyuangraph_io.h:25-187)."""
    g = _HpGraph()
    err = C.create_string_buffer(512)
    rc = _lib().hp_read_metis(path.encode(), C.byref(g), err, 512)
    if rc != 0:
        raise ValueError(f"{path}: {err.value.decode() or rc}")
    return _take(g, os.path.basename(path))


def read_mtx(path: str) -> Graph:
    """Read a square MatrixMarket coordinate matrix as the graph of its
    symmetrised pattern (diagonal dropped, unit weights); replaces the
    reference's converter matrix_to_graph/matrix_to_graph.c."""
    g = _HpGraph()
    err = C.create_string_buffer(512)
    rc = _lib().hp_read_mtx(path.encode(), C.byref(g), err, 512)
    if rc != 0:
        raise ValueError(f"{path}: {err.value.decode() or rc}")
    return _take(g, os.path.basename(path))


def mtx_to_metis(mtx_path: str, graph_path: str | None = None) -> str:
    """Convert a .mtx file to a METIS .graph file (by default next to it, with
    the extension replaced, as the reference's converter names it)."""
    if graph_path is None:
        base = mtx_path[:-4] if mtx_path.endswith(".mtx") else mtx_path
        graph_path = base + ".graph"
    g = read_mtx(mtx_path)
    write_metis(graph_path, Graph(g.xadj, g.adjncy, g.vwgt, g.adjwgt))
    return graph_path


def write_metis(path: str, g: Graph) -> None:
    h = _HpGraph(g.nvtxs, g.nedges, g.xadj.ctypes.data_as(C.POINTER(C.c_int32)),
                 g.adjncy.ctypes.data_as(C.POINTER(C.c_int32)), g.vwgt.ctypes.data_as(C.POINTER(C.c_int32)),
                 g.adjwgt.ctypes.data_as(C.POINTER(C.c_int32)))
    if _lib().hp_write_metis(path.encode(), C.byref(h)) != 0:
        raise OSError(f"cannot write {path}")


def write_partition(fname: str, part, nparts: int) -> str:
    """Write <fname>.part.<nparts> (replaces hunyuangraph_writetofile, hunyuangraph_io.h:190-205)."""
    p = np.ascontiguousarray(part, dtype=np.int32)
    if _lib().hp_write_partition(fname.encode(), p.ctypes.data_as(C.POINTER(C.c_int32)), p.shape[0],
                                 nparts) != 0:
        raise OSError(f"cannot write {fname}.part.{nparts}")
    return f"{fname}.part.{nparts}"


def set_threads(n: int) -> None:
    _lib().hp_gen_set_threads(int(n))


def grid2d(nx: int, ny: int, seed: int = 1, wmin: int = 1, wmax: int = 1) -> Graph:
    g = _HpGraph()
    _check(_lib().hp_gen_grid2d(nx, ny, seed, wmin, wmax, C.byref(g)), "hp_gen_grid2d")
    return _take(g, f"grid2d_{nx}x{ny}")


def grid3d(nx: int, ny: int, nz: int, seed: int = 2, wmin: int = 1, wmax: int = 10) -> Graph:
    g = _HpGraph()
    _check(_lib().hp_gen_grid3d(nx, ny, nz, seed, wmin, wmax, C.byref(g)), "hp_gen_grid3d")
    return _take(g, f"grid3d_{nx}x{ny}x{nz}")


def rmat(scale: int, edgefactor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 3,
         wmin: int = 1, wmax: int = 100, nvtxs_limit: int = 0) -> Graph:
    g = _HpGraph()
    _check(_lib().hp_gen_rmat(scale, edgefactor, a, b, c, seed, wmin, wmax, nvtxs_limit,
                              C.byref(g)), "hp_gen_rmat")
    return _take(g, f"rmat_s{scale}_ef{edgefactor}")


def rgg(n: int, mean_degree: float = 12.0, seed: int = 4) -> Graph:
    radius = math.sqrt(mean_degree / (math.pi * n))
    g = _HpGraph()
    _check(_lib().hp_gen_rgg(n, radius, seed, C.byref(g)), "hp_gen_rgg")
    return _take(g, f"rgg_{n}")


def edge_weight(seed: int, u: int, v: int, wmin: int, wmax: int) -> int:
    return int(_lib().hp_gen_edge_weight(seed, u, v, wmin, wmax))


def batch_specs(count: int = 1024, seed: int = 5, nmin: int = 1000, nmax: int = 200000):
    """(kind, n, k) for the uneven batch: n log-uniform in [nmin, nmax], half 2-D grids
    (nearest shape) and half R-MAT (edge factor 8), k from {2,4,8,16,32,64}."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count)).astype(np.int64)
    ks = rng.choice(np.array([2, 4, 8, 16, 32, 64]), size=count)
    specs = []
    for i in range(count):
        kind = "grid2d" if i % 2 == 0 else "rmat"
        specs.append((kind, int(ns[i]), int(ks[i])))
    return specs


def batch_graph(kind: str, n: int, seed: int) -> Graph:
    if kind == "grid2d":
        nx = max(1, int(round(math.sqrt(n))))
        ny = max(1, int(round(n / nx)))
        return grid2d(nx, ny, seed=seed, wmin=1, wmax=100)
    scale = max(1, int(math.ceil(math.log2(max(n, 2)))))
    return rmat(scale, 8, seed=seed, wmin=1, wmax=100, nvtxs_limit=n)


# The named workloads.
def config_grid2d() -> Graph:
    return grid2d(256, 256, seed=1, wmin=1, wmax=1)


def config_grid3d(side: int = 128) -> Graph:
    return grid3d(side, side, side, seed=2, wmin=1, wmax=10)


def config_rmat(scale: int = 22) -> Graph:
    return rmat(scale, 16, seed=3, wmin=1, wmax=100)


def config_rgg(n: int = 1 << 24) -> Graph:
    return rgg(n, 12.0, seed=4)


# name -> (graph constructor, nparts, imbalance factor)
WORKLOADS = {
    "grid2d": (config_grid2d, 8, 1.03),
    "grid3d": (config_grid3d, 64, 1.03),
    "rmat22": (config_rmat, 256, 1.03),
    "rmat20": (lambda: config_rmat(20), 256, 1.03),   # a quarter-size R-MAT for profiler captures
    "rgg24": (config_rgg, 1024, 1.05),
}
