"""Build the native libraries in-tree.

* ``hunyuansc25_b200/lib/libhp_b200.so`` — the partitioner (sm_100a CUDA + C++ host
  driver, C ABI in ``include/hp_partition.h``), compiled with nvcc for
  ``-gencode arch=compute_100a,code=sm_100a``.
* ``hunyuansc25_b200/lib/libhp_gen.so`` — host graph generators (``include/hp_gen.h``).

Run ``python -m hunyuansc25_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xcompiler", "-fopenmp",
]

CU_SOURCES = [
    "hp_api.cu",
    "hp_scan.cu",
    "hp_coarsen.cu",
    "hp_initpart.cu",
    "hp_refine.cu",
    "hp_mlp.cu",
    "hp_nd.cu",
]


def _run(cmd, cwd=None):
    res = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return res.stdout


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _cc():
    # a system gcc with OpenMP support (some images put a gcc without libgomp first)
    for cand in ("/usr/bin/gcc", "gcc"):
        if shutil.which(cand):
            return cand
    raise RuntimeError("gcc not found")


def build_gen(force=False):
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libhp_gen.so")
    srcs = [os.path.join(CSRC, "hp_gen.c"), os.path.join(CSRC, "hp_io.c")]
    if not force and _newer(out, srcs + [os.path.join(INCLUDE, "hp_gen.h"), os.path.join(INCLUDE, "hp_io.h")]):
        return out
    _run([_cc(), "-O2", "-fPIC", "-fopenmp", "-std=c11", "-Wall", "-I", INCLUDE, "-shared",
          "-o", out, *srcs, "-lm"])
    return out


def build_cuda(force=False, verbose_ptxas=False):
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libhp_b200.so")
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(INCLUDE, "hp_partition.h"))
    if not force and _newer(out, deps):
        return out
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    objdir = os.path.join(ROOT, "_build", "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = list(NVCC_FLAGS)
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        if force or not _newer(o, [s] + [d for d in deps if not d.endswith(".cu")]):
            log = _run([nvcc, *ARCH, *flags, "-I", INCLUDE, "-I", CSRC, "-ccbin", _cc().replace("gcc", "g++"),
                        "-c", s, "-o", o])
            if verbose_ptxas:
                sys.stderr.write(log)
        objs.append(o)
    _run([nvcc, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-ccbin", _cc().replace("gcc", "g++"),
          "-o", out, *objs, "-cudart", "static", "-lgomp"])
    return out


def build_all(force=False):
    return [build_gen(force), build_cuda(force)]


if __name__ == "__main__":
    # --ptxas: rebuild the CUDA library with ptxas's per-kernel resource report
    # (registers, shared memory, spills) on stderr
    ptxas = "--ptxas" in sys.argv
    print(build_gen(force="--force" in sys.argv))
    print(build_cuda(force="--force" in sys.argv or ptxas, verbose_ptxas=ptxas))
