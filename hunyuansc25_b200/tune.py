"""Autotuner of the kernel parameters (``hp_tuning``, include/hp_partition.h).

    python -m hunyuansc25_b200.tune --workload rmat22 [--out FILE] [--reps 3] [--sweeps 2]
    python -m hunyuansc25_b200.tune <graph.graph|matrix.mtx> <nparts> [--ub 1.03] [--out FILE]

The tuned parameters are the degree-class bounds (which kernel aggregates a
row: a thread, a lane segment, a warp, a CTA, grid-wide chunks or the dense
path), the CTAs per SM of the grid-stride kernels and the dense contraction
accumulator's bitmap layout.  They change speed only: every value in range
gives the same partition bit for bit, because each class writes the same
canonical rows and proposals.

The search times whole partitions of the graph (the library's device time,
inputs resident on the device) and walks the parameters by coordinate
descent: each parameter in turn tries its candidate values with the others
fixed and keeps the fastest when it beats the current best by more than
``min_gain``; sweeps repeat until one changes nothing.  Every candidate's
partition is compared with the default tuning's, and a difference stops the
search with TuningMismatch (it would be a kernel bug).  An interleaved
re-measurement of the defaults against the winner confirms the gain before
the winner is written to a tuning file; without a confirmed gain the file
holds the defaults.

Tuning files are JSON: ``{"format": "hp_tuning/1", "tuning": {field: value},
...}`` plus what was measured.  ``Context.load_tuning``, ``bench.py --tuning``
and the command-line partitioner's ``--tuning`` read them; the files of the
named workloads live in ``hunyuansc25_b200/tuning/<workload>.json``.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

from ._abi import TUNING_DEFAULTS, TUNING_FIELDS, default_options, tuning_violation

FORMAT = "hp_tuning/1"
TUNING_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning")

# Candidate values per parameter, in search order.  The defaults are included
# so that a parameter can return to its default in a later sweep.
SPACE = {
    "match_warp_deg": [8, 16, 24, 32, 48, 64, 128],
    "match_cta_deg": [512, 1024, 2048, 4096, 8192, 32768],
    "contract_thread_row": [8, 16, 24, 32],
    "contract_warp_row": [64, 128, 192, 256],
    "contract_cta_row": [512, 1024, 2048, 4096],
    "gain_thread_deg": [8, 16, 24, 32],
    "gain_hub_deg": [1024, 2048, 4096, 8192, 16384],
    "warp_dense_k": [0, 256, 512, 1024],
    "grid_ctas_per_sm": [2, 4, 8, 12, 16],
    "dense_sparse_ratio": [1, 2, 4, 8, 32],
    "small_level_n": [0, 2048, 4096, 8192, 16384, 32768],
    "chunk_deg": [512, 1024, 2048, 4096, 8192],
    "trial_cta_n": [128, 256, 512, 1024, 4096, 1 << 24],
    "contract_smem_cn": [0, 8192, 16384, 32768, 49152],
    "small_match_n": [0, 1024, 2048, 4096, 8192],
    "contract_hybrid": [0, 1],
    "apply_chunk_deg": [256, 512, 1024, 2048, 4096, 8192],
    "pdl": [0, 1],
    "graph_passes": [0, 1],
}


class TuningMismatch(RuntimeError):
    """A tuning changed the partition (a kernel of some row class disagrees)."""


def read_tuning_file(path: str) -> dict:
    """The full tuning stored in a tuning file (missing fields take their
    defaults); raises ValueError for a foreign format, an unknown field or a
    value out of range."""
    with open(path) as f:
        d = json.load(f)
    if d.get("format") != FORMAT:
        raise ValueError(f"{path}: not a {FORMAT} tuning file")
    stored = d.get("tuning", {})
    unknown = set(stored) - set(TUNING_FIELDS)
    if unknown:
        raise ValueError(f"{path}: unknown tuning fields {sorted(unknown)}")
    t = dict(TUNING_DEFAULTS)
    t.update({k: int(v) for k, v in stored.items()})
    bad = tuning_violation(t)
    if bad:
        raise ValueError(f"{path}: tuning field {bad} out of range")
    return t


def write_tuning_file(path: str, tuning: dict, **meta) -> None:
    bad = tuning_violation(tuning)
    if bad:
        raise ValueError(f"tuning field {bad} out of range")
    out = {"format": FORMAT, "tuning": {k: int(tuning[k]) for k in TUNING_FIELDS}}
    out.update(meta)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=False)
        f.write("\n")


def workload_tuning_path(workload: str | None, learned: bool = False) -> str | None:
    """The committed tuning file of a workload: tuning/<workload>.json for the
    plain refiner, tuning/<workload>_learned.json (when present, else the plain
    file) for the learned move proposals, whose passes move far fewer vertices
    and so favour other row-class bounds."""
    if not workload:
        return None
    if learned:
        p = os.path.join(TUNING_DIR, f"{workload}_learned.json")
        if os.path.exists(p):
            return p
    p = os.path.join(TUNING_DIR, f"{workload}.json")
    return p if os.path.exists(p) else None


def resolve_tuning(arg: str | None, workload: str | None, learned: bool = False) -> str | None:
    """Tuning file for a --tuning argument: None/'auto' -> the workload's
    committed file for that refiner if there is one, 'none' -> no file, else
    the path given."""
    if arg in (None, "auto"):
        return workload_tuning_path(workload, learned)
    if arg == "none":
        return None
    if not os.path.exists(arg):
        raise FileNotFoundError(arg)
    return arg


class Evaluator:
    """Times partitions of one resident graph under a given tuning."""

    def __init__(self, ctx, g, nparts: int, ubfactor: float, options=None, reps: int = 3, device: int = 0):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.nparts = nparts
        self.ub = ubfactor
        self.opt = options if options is not None else default_options()
        self.reps = max(1, reps)
        dev = torch.device("cuda", device)
        self.arrays = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
                       for a in (g.xadj, g.adjncy, g.vwgt, g.adjwgt)]
        self.part = torch.empty(max(g.nvtxs, 1), dtype=torch.int32, device=dev)
        self.stream = torch.cuda.Stream(dev)
        self.evaluations = 0

    def run(self, tuning: dict, reps: int | None = None):
        """(best device ms over the repetitions, partition, cut)."""
        self.ctx.set_tuning(tuning)
        xadj, adj, vw, ew = self.arrays
        times = []
        cut = None
        for _ in range(reps or self.reps):
            _, cut = self.ctx.partition_device(xadj, adj, self.nparts, vw, ew, self.ub, options=self.opt,
                                               stream=self.stream, part=self.part)
            times.append(float(self.ctx.stats().ms_total))
        self.stream.synchronize()
        self.evaluations += 1
        return min(times), self.part[:xadj.numel() - 1].cpu().numpy(), int(cut)


def autotune(ctx, g, nparts: int, ubfactor: float = 1.03, *, options=None, reps: int = 3, sweeps: int = 2,
             min_gain: float = 0.01, confirm: int = 5, space: dict | None = None, start: dict | None = None,
             log=None, device: int = 0, evaluator=None):
    """Coordinate-descent search; returns (tuning, report).  The context's
    tuning is left at the returned one.  ``evaluator`` (an object with
    ``run(tuning) -> (ms, part, cut)``, ``reps`` and ``evaluations``) replaces
    the timed partitions of ``g``."""
    space = space if space is not None else SPACE
    say = log or (lambda *_: None)
    ev = evaluator if evaluator is not None else Evaluator(ctx, g, nparts, ubfactor, options, reps, device)
    defaults = dict(TUNING_DEFAULTS)
    ev.run(defaults, reps=1)                      # warm-up (module load, arena)
    base_ms, ref_part, ref_cut = ev.run(defaults)
    best = dict(defaults)
    best.update(start or {})
    if tuning_violation(best):
        raise ValueError(f"start tuning field {tuning_violation(best)} out of range")
    best_ms = base_ms if best == defaults else ev.run(best)[0]
    say(f"defaults: {base_ms:.3f} ms, cut {ref_cut}")
    t0 = time.time()
    trail = []
    for sweep in range(max(1, sweeps)):
        changed = False
        for name, values in space.items():
            for v in values:
                if v == best[name]:
                    continue
                cand = dict(best)
                cand[name] = int(v)
                if tuning_violation(cand):
                    continue
                ms, part, cut = ev.run(cand)
                if cut != ref_cut or not np.array_equal(part, ref_part):
                    raise TuningMismatch(f"{name}={v} changed the partition (cut {cut} vs {ref_cut})")
                if ms < best_ms * (1.0 - min_gain):
                    say(f"sweep {sweep}: {name} {best[name]} -> {v}: {best_ms:.3f} -> {ms:.3f} ms")
                    trail.append({"sweep": sweep, "field": name, "value": int(v), "ms": round(ms, 3)})
                    best, best_ms, changed = cand, ms, True
        if not changed:
            break
    # interleaved confirmation: defaults and winner alternate
    d_ms, t_ms = [], []
    if best != defaults:
        for _ in range(max(1, confirm)):
            d_ms.append(ev.run(defaults)[0])
            t_ms.append(ev.run(best)[0])
        ms_default, ms_tuned = statistics.median(d_ms), statistics.median(t_ms)
        if ms_tuned > ms_default * (1.0 - min_gain / 2):
            say(f"gain not confirmed ({ms_default:.3f} vs {ms_tuned:.3f} ms): defaults kept")
            best, ms_tuned = dict(defaults), ms_default
    else:
        ms_default = ms_tuned = base_ms
    if ctx is not None:
        ctx.set_tuning(best)
    report = {
        "ms_default": round(ms_default, 3),
        "ms_tuned": round(ms_tuned, 3),
        "speedup": round(ms_default / ms_tuned, 4) if ms_tuned > 0 else None,
        "edgecut": ref_cut,
        "identical_partitions": True,
        "evaluations": ev.evaluations,
        "reps_per_evaluation": ev.reps,
        "search_seconds": round(time.time() - t0, 1),
        "changes": trail,
    }
    return best, report


def main(argv=None) -> int:
    from . import Context, graphs
    ap = argparse.ArgumentParser(prog="python -m hunyuansc25_b200.tune", description=__doc__.splitlines()[0])
    ap.add_argument("graph", nargs="?", help="METIS .graph or MatrixMarket .mtx file")
    ap.add_argument("nparts", nargs="?", type=int)
    ap.add_argument("--workload", choices=sorted(graphs.WORKLOADS))
    ap.add_argument("--ub", type=float, default=None)
    ap.add_argument("--out", default=None, help="tuning file (default: tuning/<workload>.json in the package)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--min-gain", type=float, default=0.01)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--learned", action="store_true",
                    help="tune the learned move proposals (committed weights); the file is "
                         "tuning/<workload>_learned.json")
    a = ap.parse_args(argv)
    graphs.set_threads(os.cpu_count() or 1)
    if a.workload:
        make, nparts, ub = graphs.WORKLOADS[a.workload]
        g = make()
        name = a.workload
        nparts = a.nparts or nparts
        ub = a.ub or ub
        out = a.out or os.path.join(TUNING_DIR, f"{a.workload}{'_learned' if a.learned else ''}.json")
    else:
        if not a.graph or a.nparts is None:
            ap.error("give <graph> <nparts>, or --workload")
        g = graphs.read_mtx(a.graph) if a.graph.endswith(".mtx") else graphs.read_metis(a.graph)
        name, nparts, ub = os.path.basename(a.graph), a.nparts, a.ub or 1.03
        out = a.out or f"{a.graph}.tuning.json"
    import torch
    ctx = Context(a.device)
    options = None
    if a.learned:
        from . import learn
        params, thr, _ = learn.load_params()
        ctx.mlp_set_params(params, thr)
        options = default_options(learned=1)
    best, rep = autotune(ctx, g, nparts, ub, options=options, reps=a.reps, sweeps=a.sweeps,
                         min_gain=a.min_gain, log=lambda s: print(s, flush=True), device=a.device)
    write_tuning_file(out, best, device=torch.cuda.get_device_name(a.device),
                      sm_count=torch.cuda.get_device_properties(a.device).multi_processor_count,
                      workload={"name": name, "nvtxs": g.nvtxs, "nedges_undirected": g.nedges // 2,
                                "nparts": nparts, "ubfactor": ub},
                      refiner="learned" if a.learned else "plain",
                      **rep)
    print(json.dumps({"out": out, "tuning": best, **{k: v for k, v in rep.items() if k != "changes"}}))
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
