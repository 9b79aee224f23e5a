"""ctypes mirror of include/hp_partition.h (structs, constants, prototypes)."""
from __future__ import annotations

import ctypes as C

HP_OK = 0
HP_ERR_INVALID_ARG = -1
HP_ERR_INVALID_GRAPH = -2
HP_ERR_NOMEM = -3
HP_ERR_CUDA = -4
HP_ERR_TIMEOUT = -5
HP_ERR_NO_DEVICE = -6
HP_ERR_UNSUPPORTED = -7
HP_ERR_INTERNAL = -8
HP_MAX_PARTS = 16384
HP_OPTIONS_VERSION = 1
HP_SCAN_NOALLOC_MAX_N = 1 << 26
HP_MLP_NPARAM = 1377
HP_PROF_NCLASS = 12

HP_TRACE_XADJ = 0
HP_TRACE_ADJNCY = 1
HP_TRACE_ADJWGT = 2
HP_TRACE_VWGT = 3
HP_TRACE_MATCH = 4
HP_TRACE_CMAP = 5
HP_TRACE_WHERE_START = 6
HP_TRACE_WHERE_FINAL = 7

ERROR_NAMES = {
    HP_OK: "HP_OK",
    HP_ERR_INVALID_ARG: "HP_ERR_INVALID_ARG",
    HP_ERR_INVALID_GRAPH: "HP_ERR_INVALID_GRAPH",
    HP_ERR_NOMEM: "HP_ERR_NOMEM",
    HP_ERR_CUDA: "HP_ERR_CUDA",
    HP_ERR_TIMEOUT: "HP_ERR_TIMEOUT",
    HP_ERR_NO_DEVICE: "HP_ERR_NO_DEVICE",
    HP_ERR_UNSUPPORTED: "HP_ERR_UNSUPPORTED",
    HP_ERR_INTERNAL: "HP_ERR_INTERNAL",
}


class HpOptions(C.Structure):
    _fields_ = [
        ("version", C.c_int32),
        ("coarsen_to", C.c_int32),
        ("match_rounds", C.c_int32),
        ("refine_patience", C.c_int32),
        ("init_starts", C.c_int32),
        ("fm_passes", C.c_int32),
        ("max_levels", C.c_int32),
        ("learned", C.c_int32),
        ("validate", C.c_int32),
        ("trace", C.c_int32),
        ("profile", C.c_int32),
        ("eager", C.c_int32),
        ("seed", C.c_uint64),
    ]


def default_options(**overrides) -> HpOptions:
    """Same defaults as hp_options_default() (checked by a test)."""
    o = HpOptions()
    o.version = HP_OPTIONS_VERSION
    o.coarsen_to = 0
    o.match_rounds = 6
    o.refine_patience = 5
    o.init_starts = 256
    o.fm_passes = 10
    o.max_levels = 64
    o.learned = 0
    o.validate = 1
    o.trace = 0
    o.profile = 0
    o.eager = 0
    o.seed = 1
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


TUNING_FIELDS = [
    "match_warp_deg",
    "match_cta_deg",
    "contract_thread_row",
    "contract_warp_row",
    "contract_cta_row",
    "gain_thread_deg",
    "gain_hub_deg",
    "warp_dense_k",
    "grid_ctas_per_sm",
    "dense_sparse_ratio",
    "small_level_n",
    "chunk_deg",
    "trial_cta_n",
    "contract_smem_cn",
    "batch_workers",
    "small_match_n",
    "contract_hybrid",
    "apply_chunk_deg",
    "pdl",
    "graph_passes",
]

TUNING_DEFAULTS = {
    "match_warp_deg": 32,
    "match_cta_deg": 4096,
    "contract_thread_row": 32,
    "contract_warp_row": 256,
    "contract_cta_row": 4096,
    "gain_thread_deg": 32,
    "gain_hub_deg": 4096,
    "warp_dense_k": 1024,
    "grid_ctas_per_sm": 8,
    "dense_sparse_ratio": 4,
    "small_level_n": 4096,
    "chunk_deg": 4096,
    "trial_cta_n": 512,
    "contract_smem_cn": 49152,
    "batch_workers": 16,
    "small_match_n": 8192,
    "contract_hybrid": 1,
    "apply_chunk_deg": 4096,
    "pdl": 1,
    "graph_passes": 1,
}

TUNE_DEG_MAX = 1 << 24


def tuning_violation(t: dict):
    """First field of a tuning out of range, else None (the ranges that
    hp_context_set_tuning checks)."""
    lim = [
        ("match_warp_deg", 4, 256),
        ("match_cta_deg", t["match_warp_deg"], TUNE_DEG_MAX),
        ("contract_thread_row", 8, 32),
        ("contract_warp_row", t["contract_thread_row"], 256),
        ("contract_cta_row", t["contract_warp_row"], 4096),
        ("gain_thread_deg", 8, 32),
        ("gain_hub_deg", t["gain_thread_deg"], TUNE_DEG_MAX),
        ("warp_dense_k", 0, 1024),
        ("grid_ctas_per_sm", 1, 32),
        ("dense_sparse_ratio", 1, 4096),
        ("small_level_n", 0, 32768),
        ("chunk_deg", t["gain_thread_deg"], TUNE_DEG_MAX),
        ("trial_cta_n", 1, TUNE_DEG_MAX),
        ("contract_smem_cn", 0, 49152),
        ("batch_workers", 1, 64),
        ("small_match_n", 0, 8192),
        ("contract_hybrid", 0, 1),
        ("apply_chunk_deg", t["gain_thread_deg"], TUNE_DEG_MAX),
        ("pdl", 0, 1),
        ("graph_passes", 0, 1),
    ]
    for name, lo, hi in lim:
        if not lo <= int(t[name]) <= hi:
            return name
    return None


class HpTuning(C.Structure):
    _fields_ = [(name, C.c_int32) for name in TUNING_FIELDS] + [("reserved", C.c_int32 * 4)]

    @classmethod
    def from_dict(cls, d: dict) -> "HpTuning":
        unknown = set(d) - set(TUNING_FIELDS)
        if unknown:
            raise ValueError(f"unknown tuning fields: {sorted(unknown)}")
        t = cls()
        for name in TUNING_FIELDS:
            setattr(t, name, int(d.get(name, TUNING_DEFAULTS[name])))
        return t

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name in TUNING_FIELDS}


class HpStats(C.Structure):
    _fields_ = [
        ("edgecut", C.c_int64),
        ("max_excess", C.c_int64),
        ("tvwgt", C.c_int64),
        ("nlevels", C.c_int32),
        ("coarsest_nvtxs", C.c_int32),
        ("coarsest_nedges", C.c_int64),
        ("refine_passes", C.c_int32),
        ("kernel_launches", C.c_int32),
        ("ms_total", C.c_float),
        ("ms_coarsen", C.c_float),
        ("ms_init", C.c_float),
        ("ms_uncoarsen", C.c_float),
        ("ms_h2d", C.c_float),
        ("ms_d2h", C.c_float),
        ("prof_ms", C.c_float * HP_PROF_NCLASS),
        ("prof_bytes", C.c_int64 * HP_PROF_NCLASS),
        ("prof_launches", C.c_int32 * HP_PROF_NCLASS),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name.startswith("prof_") else v
        return out


HP_PROF_MATCH = 0
HP_PROF_CONTRACT = 1
HP_PROF_GAIN = 2
HP_PROF_LP = 3
HP_PROF_REBUILD = 4
HP_PROF_INIT = 5
HP_PROF_MATCH_MORE = 6
HP_PROF_REBALANCE = 7
HP_PROF_APPLY = 8
# class names by index; "" for the unused slots of the stats arrays
PROF_NAMES = ["match", "contract", "gain_build", "lp", "rebuild", "init_trials", "match_more", "rebalance",
              "apply", "", "", ""]


I32P = C.POINTER(C.c_int32)
I64P = C.POINTER(C.c_int64)
F32P = C.POINTER(C.c_float)

# name -> (restype, argtypes); every symbol include/hp_partition.h declares.
PROTOTYPES = {
    "hp_options_default": (None, [C.POINTER(HpOptions)]),
    "hp_strerror": (C.c_char_p, [C.c_int]),
    "hp_tuning_default": (None, [C.POINTER(HpTuning)]),
    "hp_context_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(HpTuning)]),
    "hp_context_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(HpTuning)]),
    "hp_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "hp_context_destroy": (None, [C.c_void_p]),
    "hp_partition": (C.c_int, [C.c_void_p, C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, F32P,
                               C.c_float, C.POINTER(HpOptions), I32P, I64P]),
    "hp_partition_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int32, F32P, C.c_float,
                                      C.POINTER(HpOptions), C.c_void_p, C.c_void_p, I64P]),
    "hp_last_stats": (C.c_int, [C.c_void_p, C.POINTER(HpStats)]),
    "hp_trace_nlevels": (C.c_int, [C.c_void_p]),
    "hp_trace_level": (C.c_int, [C.c_void_p, C.c_int, I32P, I64P, I64P, I64P]),
    "hp_trace_copy": (C.c_int, [C.c_void_p, C.c_int, C.c_int, I32P, C.c_int64]),
    "hp_partition_batch": (C.c_int, [C.c_void_p, C.c_int32, I64P, I64P, I32P, I32P, I32P, I32P,
                                     I32P, F32P, C.POINTER(HpOptions), I32P, I64P]),
    "hp_mlp_set_params": (C.c_int, [C.c_void_p, F32P, C.c_int32, C.c_float]),
    "hp_mlp_get_params": (C.c_int, [C.c_void_p, F32P, C.c_int32]),
    "hp_mlp_loss_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, F32P, F32P]),
    "hp_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32,
                               C.c_int32, C.c_float, F32P]),
    "hp_mlp_infer": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32]),
    "hp_movelog_enable": (C.c_int, [C.c_void_p, C.c_int64]),
    "hp_movelog_count": (C.c_int64, [C.c_void_p]),
    "hp_movelog_copy": (C.c_int, [C.c_void_p, F32P, F32P, C.c_int64]),
    "hp_movelog_reset": (C.c_int, [C.c_void_p]),
    "hp_node_nd": (C.c_int, [C.c_void_p, C.c_int32, I32P, I32P, I32P, C.POINTER(HpOptions), I32P, I32P]),
    "hp_scan_exclusive_i32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                        C.c_void_p]),
    "hp_scan_exclusive_i32_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "hp_test_wait_expiry": (C.c_int, [C.c_void_p]),
    "hp_test_arena_first": (C.c_int, [C.c_void_p, C.c_int64]),
    "hp_test_arena_restarts": (C.c_int, [C.c_void_p]),
    "hp_edgecut_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, I64P]),
    "hunyuangraph_PartitionGraph": (None, [I32P, I32P, I32P, I32P, I32P, I32P, F32P, F32P, I32P]),
}
