"""ctypes binding of the C ABI in include/bv_pairhmm.h.

The shared library is built in-tree (biovoltron_b200/_native/libbv_pairhmm.so,
``make -C biovoltron_b200/csrc``).  There is no fallback: if the library is
missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_native", "libbv_pairhmm.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "bv_pairhmm.h")

BV_OK = 0
BV_ERR_INVALID_ARG = 1
BV_ERR_OOM = 2
BV_ERR_CUDA = 3
BV_ERR_TIMEOUT = 4
BV_ERR_NO_DEVICE = 5
BV_ERR_INTERNAL = 6
BV_ERR_UNSUPPORTED = 7

BV_PRECISION_AUTO = 0
BV_PRECISION_F64 = 1
BV_MODE_FULL = 0
BV_MODE_BAND = 1


class Options(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("device", C.c_int32), ("precision", C.c_int32), ("mode", C.c_int32),
        ("rescue_threshold", C.c_double), ("haps_per_unit", C.c_int32), ("haps_per_warp", C.c_int32),
        ("pipeline_chunks", C.c_int32), ("pipeline_min_pairs", C.c_int32), ("reserved", C.c_int32 * 4),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("pairs", C.c_int64), ("cells", C.c_int64), ("rescued", C.c_int64), ("underflow", C.c_int64),
        ("band_pairs", C.c_int64), ("band_fallback", C.c_int64), ("band_cells", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("ms_h2d", C.c_double), ("ms_fp32", C.c_double), ("ms_fp64", C.c_double), ("ms_band", C.c_double),
        ("ms_d2h", C.c_double), ("ms_total", C.c_double),
        ("band_routed_full", C.c_int64), ("audit_pairs", C.c_int64), ("audit_max_err", C.c_double),
        ("audit_p99_err", C.c_double), ("band_promoted", C.c_int64), ("ms_seed", C.c_double),
        ("ms_full", C.c_double), ("rescued_cells", C.c_int64), ("band_result_cells", C.c_int64),
        ("fp32_skipped_cells", C.c_int64), ("band_rescored", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BandOptions(C.Structure):
    _fields_ = [("struct_size", C.c_int32), ("enabled", C.c_int32), ("use_mlp", C.c_int32),
                ("fixed_half", C.c_int32), ("margin", C.c_int32), ("audit_period", C.c_int32),
                ("edge_threshold", C.c_double), ("cap_margin", C.c_float), ("reserved", C.c_int32 * 5)]


class BandTrainOptions(C.Structure):
    _fields_ = [("struct_size", C.c_int32), ("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float),
                ("alpha", C.c_float), ("tau", C.c_float), ("clip", C.c_float), ("margin", C.c_int32),
                ("seed", C.c_uint64), ("reserved", C.c_int32 * 4)]


class BandTrainReport(C.Structure):
    _fields_ = [("pairs", C.c_int64), ("labelled", C.c_int64), ("steps", C.c_int32), ("first_loss", C.c_float),
                ("last_loss", C.c_float), ("cover_frac", C.c_double), ("band_frac", C.c_double),
                ("ms_labels", C.c_double), ("ms_train", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneEntry(C.Structure):
    _fields_ = [("rows_per_lane", C.c_int32), ("haps_per_warp", C.c_int32), ("warps_per_block", C.c_int32),
                ("reserved", C.c_int32), ("ms", C.c_double)]

    def as_dict(self):
        return {"rows_per_lane": self.rows_per_lane, "haps_per_warp": self.haps_per_warp,
                "warps_per_block": self.warps_per_block, "ms": self.ms}


class TestcaseC(C.Structure):
    _fields_ = [
        ("rslen", C.c_int), ("haplen", C.c_int),
        ("q", C.c_void_p), ("i", C.c_void_p), ("d", C.c_void_p), ("c", C.c_void_p),
        ("hap", C.c_void_p), ("rs", C.c_void_p),
    ]


class ShaccRead(C.Structure):
    _fields_ = [("length", C.c_int), ("bases", C.c_void_p), ("q", C.c_void_p), ("i", C.c_void_p),
                ("d", C.c_void_p), ("c", C.c_void_p)]


class ShaccHap(C.Structure):
    _fields_ = [("length", C.c_int), ("bases", C.c_void_p)]


class ShaccBatch(C.Structure):
    _fields_ = [("num_reads", C.c_int), ("num_haps", C.c_int), ("num_cells", C.c_long),
                ("reads", C.POINTER(ShaccRead)), ("haps", C.POINTER(ShaccHap)), ("results", C.POINTER(C.c_float))]


class RegionBatchC(C.Structure):
    _fields_ = [
        ("num_regions", C.c_int64), ("region_reads", C.c_void_p), ("region_haps", C.c_void_p),
        ("num_reads", C.c_int64), ("read_offsets", C.c_void_p),
        ("read_bases", C.c_void_p), ("read_q", C.c_void_p), ("read_i", C.c_void_p), ("read_d", C.c_void_p),
        ("read_c", C.c_void_p),
        ("num_haps", C.c_int64), ("hap_offsets", C.c_void_p), ("hap_bases", C.c_void_p),
        ("gap_ins", C.c_uint8), ("gap_del", C.c_uint8), ("gap_gcp", C.c_uint8), ("reserved_", C.c_uint8 * 5),
    ]


class GenotypeBatch(C.Structure):
    _fields_ = [("allele_count", C.c_void_p), ("hap_allele", C.c_void_p), ("read_overlaps", C.c_void_p)]


class NativeError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"bv_pairhmm status {status}: {msg}")
        self.status = status


_lib = None


def load() -> C.CDLL:
    """Loads the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built; run `make -C biovoltron_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    P, V = C.POINTER, C.c_void_p
    sig = {
        "bv_phmm_default_options": (None, [P(Options)]),
        "bv_phmm_abi_version": (C.c_int, []),
        "bv_phmm_status_string": (C.c_char_p, [C.c_int]),
        "bv_phmm_create": (C.c_int, [P(Options), P(V)]),
        "bv_phmm_destroy": (None, [V]),
        "bv_phmm_last_error": (C.c_char_p, [V]),
        "bv_phmm_compute_testcases": (C.c_int, [V, P(TestcaseC), C.c_int64, V, P(Stats)]),
        "bv_phmm_shacc_calculate": (C.c_int, [V, P(ShaccBatch)]),
        "bv_phmm_region_results": (C.c_int64, [P(RegionBatchC)]),
        "bv_phmm_compute_regions": (C.c_int, [V, P(RegionBatchC), V, P(Stats)]),
        "bv_phmm_stage_regions": (C.c_int, [V, P(RegionBatchC)]),
        "bv_phmm_run_staged": (C.c_int, [V, P(Stats)]),
        "bv_phmm_fetch_results": (C.c_int, [V, V, C.c_int64]),
        "bv_phmm_host_register": (C.c_int, [V, V, C.c_size_t]),
        "bv_phmm_host_unregister": (C.c_int, [V, V]),
        "bv_phmm_debug_tables": (C.c_int, [V, V, V, V, C.c_int]),
        "bv_phmm_default_band_options": (None, [P(BandOptions)]),
        "bv_phmm_set_band_options": (C.c_int, [V, P(BandOptions)]),
        "bv_phmm_measure_fp32_peak": (C.c_int, [C.c_int, P(C.c_double)]),
        "bv_phmm_measure_fp64_peak": (C.c_int, [C.c_int, P(C.c_double)]),
        "bv_phmm_default_band_train_options": (None, [P(BandTrainOptions)]),
        "bv_phmm_band_train": (C.c_int, [V, P(RegionBatchC), P(BandTrainOptions), P(BandTrainReport)]),
        "bv_phmm_band_labels": (C.c_int, [V, P(RegionBatchC), C.c_float, V, V, V, V, V, V]),
        "bv_phmm_band_routes": (C.c_int, [V, C.c_int64, V, V, V]),
        "bv_phmm_band_param_count": (C.c_int64, []),
        "bv_phmm_band_get_weights": (C.c_int, [V, V, C.c_int64]),
        "bv_phmm_band_set_weights": (C.c_int, [V, V, C.c_int64]),
        "bv_phmm_band_save": (C.c_int, [V, C.c_char_p]),
        "bv_phmm_band_load": (C.c_int, [V, C.c_char_p]),
        "bv_phmm_band_mlp_eval": (C.c_int, [V, V, V, V, C.c_int64, C.c_float, V, V, V]),
        "bv_phmm_band_mlp_infer": (C.c_int, [V, V, C.c_int64, V]),
        "bv_phmm_autotune": (C.c_int, [V, P(RegionBatchC), C.c_int32, P(TuneEntry), P(C.c_int32)]),
        "bv_phmm_set_tuning": (C.c_int, [V, P(TuneEntry), C.c_int32]),
        "bv_phmm_get_tuning": (C.c_int, [V, P(TuneEntry), P(C.c_int32)]),
        "bv_phmm_set_transitions": (C.c_int, [V, P(C.c_double)]),
        "bv_phmm_genotype_staged": (C.c_int, [V, P(RegionBatchC), P(GenotypeBatch), V, V, V, V, P(C.c_double)]),
        "bv_phmm_debug_jacobian_table": (C.c_int, [V, C.c_int]),
        "bv_phmm_debug_chunks": (C.c_int64, [P(RegionBatchC), C.c_int32, V, C.c_int64]),
        "bv_phmm_set_long_warps": (C.c_int, [V, C.c_int32]),
        "bv_phmm_get_long_warps": (C.c_int32, [V]),
        "bv_phmm_autotune_long": (C.c_int, [V, P(RegionBatchC), C.c_int32, V, V]),
        "bv_phmm_get_transitions": (C.c_int, [V, P(C.c_double)]),
        "bv_phmm_plan_partition": (C.c_int64, [P(RegionBatchC), C.c_int32, C.c_int32, V, V, V]),
        "bv_phmm_compute_regions_multi": (C.c_int, [P(V), C.c_int32, P(RegionBatchC), V, P(Stats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def header_functions(path: str = HEADER_PATH) -> List[str]:
    """Names of the functions declared in the C ABI header."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bv_phmm_[a-z0-9_]+)\s*\(", txt)))
