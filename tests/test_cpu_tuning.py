"""Kernel tuning on the host: the hp_tuning layout against the C header, the
library's defaults, tuning files, and the autotuner's search logic (with a
scripted evaluator in place of timed partitions)."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from hunyuansc25_b200 import _abi, tune
from hunyuansc25_b200._abi import TUNING_DEFAULTS, TUNING_FIELDS, HpTuning, tuning_violation

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tuning_struct_matches_header(tmp_path):
    src = tmp_path / "t.c"
    fields = " ".join(f'printf("%zu ", offsetof(hp_tuning, {f}));' for f in TUNING_FIELDS)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "hp_partition.h"\n'
                   'int main(void) {' + fields + ' printf("%zu %zu\\n", offsetof(hp_tuning, reserved), '
                   'sizeof(hp_tuning)); return 0; }\n')
    exe = tmp_path / "t"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [getattr(HpTuning, f).offset for f in TUNING_FIELDS] + [HpTuning.reserved.offset, C.sizeof(HpTuning)]
    assert got == want
    assert C.sizeof(HpTuning) == 96


def test_library_defaults_match_python():
    from hunyuansc25_b200 import load_library
    lib = load_library()
    t = HpTuning()
    lib.hp_tuning_default(C.byref(t))
    assert t.as_dict() == TUNING_DEFAULTS
    assert list(t.reserved) == [0] * 4
    assert tuning_violation(TUNING_DEFAULTS) is None


@pytest.mark.parametrize("field,value", [
    ("match_warp_deg", 3), ("match_warp_deg", 257), ("match_cta_deg", 16), ("contract_thread_row", 33),
    ("contract_thread_row", 7), ("contract_warp_row", 257), ("contract_cta_row", 4097), ("contract_cta_row", 100),
    ("gain_thread_deg", 33), ("gain_hub_deg", 31), ("warp_dense_k", 1025), ("warp_dense_k", -1),
    ("grid_ctas_per_sm", 0), ("grid_ctas_per_sm", 33), ("dense_sparse_ratio", 0),
    ("small_level_n", -1), ("small_level_n", 32769), ("chunk_deg", 31), ("trial_cta_n", 0), ("contract_smem_cn", 49153),
    ("batch_workers", 0), ("batch_workers", 65), ("small_match_n", -1), ("small_match_n", 8193),
    ("contract_hybrid", -1), ("contract_hybrid", 2), ("apply_chunk_deg", 31),
])
def test_violations(field, value):
    t = dict(TUNING_DEFAULTS)
    t[field] = value
    assert tuning_violation(t) == field


def test_every_search_value_is_in_range_alone():
    for name, values in tune.SPACE.items():
        assert TUNING_DEFAULTS[name] in values, name
        for v in values:
            t = dict(TUNING_DEFAULTS)
            t[name] = v
            # a value may conflict with the default of a related bound only
            # where the ordered bounds allow it
            bad = tuning_violation(t)
            assert bad in (None, name), (name, v, bad)


def test_tuning_file_round_trip(tmp_path):
    t = dict(TUNING_DEFAULTS, match_warp_deg=16, grid_ctas_per_sm=4)
    p = tmp_path / "x.json"
    tune.write_tuning_file(str(p), t, ms_default=1.0, ms_tuned=0.9)
    assert tune.read_tuning_file(str(p)) == t
    d = json.loads(p.read_text())
    assert d["format"] == tune.FORMAT and d["ms_tuned"] == 0.9
    # partial files take the defaults for the missing fields
    p.write_text(json.dumps({"format": tune.FORMAT, "tuning": {"warp_dense_k": 256}}))
    assert tune.read_tuning_file(str(p)) == dict(TUNING_DEFAULTS, warp_dense_k=256)


@pytest.mark.parametrize("body,msg", [
    ({"format": "other", "tuning": {}}, "not a"),
    ({"format": tune.FORMAT, "tuning": {"bogus": 1}}, "unknown"),
    ({"format": tune.FORMAT, "tuning": {"warp_dense_k": 5000}}, "out of range"),
])
def test_tuning_file_rejects(tmp_path, body, msg):
    p = tmp_path / "bad.json"
    p.write_text(json.dumps(body))
    with pytest.raises(ValueError, match=msg):
        tune.read_tuning_file(str(p))


def test_committed_tuning_files_are_valid():
    if not os.path.isdir(tune.TUNING_DIR):
        pytest.skip("no committed tuning files")
    names = [f for f in os.listdir(tune.TUNING_DIR) if f.endswith(".json")]
    for f in names:
        t = tune.read_tuning_file(os.path.join(tune.TUNING_DIR, f))
        assert tuning_violation(t) is None


def test_resolve_tuning(tmp_path):
    assert tune.resolve_tuning("none", "grid3d") is None
    assert tune.resolve_tuning("auto", "no_such_workload") is None
    assert tune.resolve_tuning(None, None) is None
    p = tmp_path / "t.json"
    tune.write_tuning_file(str(p), TUNING_DEFAULTS)
    assert tune.resolve_tuning(str(p), "grid3d") == str(p)
    with pytest.raises(FileNotFoundError):
        tune.resolve_tuning(str(tmp_path / "missing.json"), None)


class ScriptedEvaluator:
    """Deterministic cost model: each field contributes |value - optimum|."""

    def __init__(self, optimum, change_partition=None):
        self.optimum = optimum
        self.change_partition = change_partition or {}
        self.reps = 1
        self.evaluations = 0
        self.seen = []

    def run(self, tuning, reps=None):
        self.evaluations += 1
        self.seen.append(dict(tuning))
        ms = 10.0 + sum(abs(tuning[k] - v) / (1.0 + abs(v)) for k, v in self.optimum.items())
        part = np.zeros(8, np.int32)
        for k, v in self.change_partition.items():
            if tuning[k] == v:
                part[0] = 1
        return ms, part, 7


def test_coordinate_descent_finds_the_separable_optimum():
    opt = {"match_warp_deg": 16, "grid_ctas_per_sm": 4, "warp_dense_k": 512}
    ev = ScriptedEvaluator(opt)
    best, rep = tune.autotune(None, None, 8, evaluator=ev, min_gain=0.001, confirm=1)
    for k, v in opt.items():
        assert best[k] == v
    for k in TUNING_FIELDS:
        if k not in opt:
            assert best[k] == TUNING_DEFAULTS[k]
    assert rep["ms_tuned"] < rep["ms_default"]
    assert rep["identical_partitions"]
    assert all(tuning_violation(t) is None for t in ev.seen)


def test_no_gain_keeps_defaults():
    ev = ScriptedEvaluator({k: TUNING_DEFAULTS[k] for k in ("match_warp_deg",)})
    best, rep = tune.autotune(None, None, 8, evaluator=ev, confirm=1)
    assert best == TUNING_DEFAULTS
    assert rep["speedup"] == 1.0


def test_partition_change_is_reported():
    ev = ScriptedEvaluator({"grid_ctas_per_sm": 4}, change_partition={"grid_ctas_per_sm": 2})
    with pytest.raises(tune.TuningMismatch, match="grid_ctas_per_sm"):
        tune.autotune(None, None, 8, evaluator=ev)


def test_prototypes_cover_tuning_symbols():
    for name in ("hp_tuning_default", "hp_context_set_tuning", "hp_context_get_tuning"):
        assert name in _abi.PROTOTYPES
