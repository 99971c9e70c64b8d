"""ctypes binding of libkestrel_gpu.so (the C ABI in include/kestrel_gpu.h).

The library is the only compute path: if it is missing or no CUDA device is
present, calls raise instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkestrel_gpu.so")

KG_OK, KG_EINVAL, KG_ENOMEM, KG_ECUDA, KG_ETIMEOUT, KG_ENOSITES, KG_ENOTREADY, KG_ENOTFOUND, \
    KG_ECANCELED = range(9)
KG_PREC_FP32C, KG_PREC_FP64 = 0, 1
MISSING = 3

STATUS_NAMES = {0: "KG_OK", 1: "KG_EINVAL", 2: "KG_ENOMEM", 3: "KG_ECUDA", 4: "KG_ETIMEOUT",
                5: "KG_ENOSITES", 6: "KG_ENOTREADY", 7: "KG_ENOTFOUND", 8: "KG_ECANCELED"}


class KgOutput(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint64), ("y", ctypes.c_uint64),
                ("jacquard", ctypes.c_double * 9), ("obj", ctypes.c_double),
                ("iters", ctypes.c_uint64), ("cond", ctypes.c_double)]


class KgCohort(ctypes.Structure):
    _fields_ = [("codes", ctypes.c_void_p), ("n_samples", ctypes.c_int64),
                ("n_sites", ctypes.c_int64), ("row_stride", ctypes.c_int64),
                ("allele_frequencies", ctypes.c_void_p), ("num_samples", ctypes.c_int64),
                ("out", ctypes.c_void_p), ("out_cap", ctypes.c_int64),
                ("n_out", ctypes.c_int64), ("status", ctypes.c_int32)]


class KgRunStats(ctypes.Structure):
    _fields_ = [("gh_passes", ctypes.c_uint64), ("obj_passes", ctypes.c_uint64),
                ("fp64_passes", ctypes.c_uint64), ("fp64_pairs", ctypes.c_uint64),
                ("pair_sites", ctypes.c_uint64), ("work_units", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("flops_fp32", ctypes.c_uint64),
                ("flops_fp64", ctypes.c_uint64), ("shape_sites", ctypes.c_uint64 * 5),
                ("nonconverged", ctypes.c_uint64),
                ("waves", ctypes.c_uint64), ("slots", ctypes.c_uint64),
                ("admit_ms", ctypes.c_double), ("pass_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("pair_kernel_ms", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("sites_used", ctypes.c_uint64 * 3),
                ("sites_discarded", ctypes.c_uint64)]


OUTPUT_DTYPE = np.dtype([("x", np.uint64), ("y", np.uint64), ("jacquard", np.float64, 9),
                         ("obj", np.float64), ("iters", np.uint64), ("cond", np.float64)])
assert OUTPUT_DTYPE.itemsize == ctypes.sizeof(KgOutput) == 112

# Every symbol include/kestrel_gpu.h declares.
EXPORTS = ("kg_create", "kg_destroy", "kg_last_error", "kg_version", "kg_set_precision",
           "kg_set_launch", "kg_set_wave_limit", "kg_set_work_unit", "kg_get_launch", "kg_autotune", "kg_load_genotypes", "kg_load_genotypes_2bit",
           "kg_set_allele_frequencies", "kg_load_multiallelic", "kg_load_likelihoods", "kg_load_likelihoods_multiallelic", "kg_relatedness_gl",
           "kg_relatedness", "kg_relatedness_gt", "kg_relatedness_coefficients",
           "kg_relatedness_batch", "kg_panel_load", "kg_submit", "kg_poll", "kg_wait",
           "kg_cancel", "kg_serving_stats", "kg_relatedness_noalloc", "kg_last_run_stats",
           "kg_fp32_peak", "kg_run_cli", "kg_vcf_read", "kg_vcf_error", "kg_vcf_info", "kg_vcf_codes",
           "kg_vcf_codes_2bit", "kg_vcf_likelihoods", "kg_vcf_likelihoods_multiallelic", "kg_vcf_multiallelic", "kg_vcf_sample", "kg_vcf_free")


class KestrelError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib():
    """Loads libkestrel_gpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m kestrel_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, i64, u64, i32, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
    sig = {
        "kg_create": ([ctypes.POINTER(P), i32, ctypes.c_size_t], i32),
        "kg_destroy": ([P], i32),
        "kg_last_error": ([P], ctypes.c_char_p),
        "kg_version": ([], ctypes.c_char_p),
        "kg_set_precision": ([P, i32], i32),
        "kg_set_launch": ([P, i32, i32], i32),
        "kg_set_wave_limit": ([P, u64], i32),
        "kg_set_work_unit": ([P, i32], i32),
        "kg_get_launch": ([P, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32)],
                          i32),
        "kg_autotune": ([P, ctypes.POINTER(i32), ctypes.POINTER(i32)], i32),
        "kg_load_genotypes": ([P, P, i64, i64, i64], i32),
        "kg_load_genotypes_2bit": ([P, P, P, i64, i64], i32),
        "kg_set_allele_frequencies": ([P, P], i32),
        "kg_load_multiallelic": ([P, P, i64, i64, i64, P, P], i32),
        "kg_load_likelihoods": ([P, P, i64, i64], i32),
        "kg_load_likelihoods_multiallelic": ([P, P, i64, i64, i32], i32),
        "kg_relatedness_gl": ([P, i64, u64, ctypes.c_double, P, i64, ctypes.POINTER(i64)], i32),
        "kg_relatedness": ([P, i64, u64, dbl, P, i64, ctypes.POINTER(i64)], i32),
        "kg_relatedness_gt": ([P, i64, u64, P, i64, ctypes.POINTER(i64)], i32),
        "kg_relatedness_coefficients": ([P, i64, i64, i64, P, i64, u64, dbl, i64, P, i64,
                                         ctypes.POINTER(i64)], i32),
        "kg_relatedness_batch": ([P, P, i32, u64, dbl], i32),
        "kg_panel_load": ([P, P, i64, i64, i64, P, dbl], i32),
        "kg_submit": ([P, P, i64, i64, P, u64, ctypes.POINTER(i64)], i32),
        "kg_poll": ([P, i64, ctypes.POINTER(i32)], i32),
        "kg_wait": ([P, i64, i64, P, i64, ctypes.POINTER(i64)], i32),
        "kg_cancel": ([P, i64], i32),
        "kg_serving_stats": ([P, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i64)], i32),
        "kg_last_run_stats": ([P, ctypes.POINTER(KgRunStats)], i32),
        "kg_relatedness_noalloc": ([P, i64, i64, i64, u64, dbl, P, i64, P], i32),
        "kg_fp32_peak": ([i32, ctypes.POINTER(dbl)], i32),
        "kg_run_cli": ([i32, ctypes.POINTER(ctypes.c_char_p)], i32),
        "kg_vcf_read": ([ctypes.c_char_p, ctypes.c_char_p, i32, i32, ctypes.POINTER(P)], i32),
        "kg_vcf_error": ([P], ctypes.c_char_p),
        "kg_vcf_info": ([P, ctypes.POINTER(i64), ctypes.POINTER(i64), P], i32),
        "kg_vcf_codes": ([P, P, P], i32),
        "kg_vcf_multiallelic": ([P, P, P, P], i32),
        "kg_vcf_codes_2bit": ([P, P, P], i32),
        "kg_vcf_likelihoods": ([P, P], i32),
        "kg_vcf_likelihoods_multiallelic": ([P, i32, P], i32),
        "kg_vcf_sample": ([P, i64], ctypes.c_char_p),
        "kg_vcf_free": ([P], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)
