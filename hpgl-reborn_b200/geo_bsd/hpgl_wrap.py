"""ctypes binding of libhpgl_b200.so (include/hpgl_b200.h).

Struct layouts are those of the reference's binding (src/geo_bsd/hpgl_wrap.py:44-165)
so code written against HPGL's ctypes structs keeps working. The library is
loaded from this package's directory; there is no CPU fallback: a missing or
unloadable library raises ImportError at import time.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
from numpy.ctypeslib import ndpointer

hpgl_output_handler = C.CFUNCTYPE(C.c_int, C.c_char_p, C.py_object)
hpgl_progress_handler = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_int, C.py_object)


class _HPGL_SHAPE(C.Structure):
    _fields_ = [("data", C.c_int * 3), ("strides", C.c_int * 3)]


class _HPGL_CONT_MASKED_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_ubyte)), ("shape", _HPGL_SHAPE)]


class _HPGL_IND_MASKED_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("mask", C.POINTER(C.c_ubyte)), ("shape", _HPGL_SHAPE),
                ("indicator_count", C.c_int)]


class _HPGL_KRIGING_KIND:
    ordinary = 0
    simple = 1


class _HPGL_UBYTE_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("shape", _HPGL_SHAPE)]


class _HPGL_FLOAT_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("shape", _HPGL_SHAPE)]


class _HPGL_OK_PARAMS(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int)]


class _HPGL_SK_PARAMS(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("automatic_mean", C.c_ubyte), ("mean", C.c_double)]


class _HPGL_MEDIAN_IK_PARAMS(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("marginal_probs", C.c_double * 2)]


class _HPGL_IK_PARAMS(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("marginal_prob", C.c_double)]


class __hpgl_cov_params_t(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double)]


_HPGL_COV_PARAMS = __hpgl_cov_params_t


class __hpgl_cockriging_m1_params_t(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("primary_mean", C.c_double), ("secondary_mean", C.c_double),
                ("secondary_variance", C.c_double), ("correlation_coef", C.c_double)]


class __hpgl_cockriging_m2_params_t(C.Structure):
    _fields_ = [("primary_cov_params", _HPGL_COV_PARAMS), ("secondary_cov_params", _HPGL_COV_PARAMS),
                ("radiuses", C.c_int * 3), ("max_neighbours", C.c_int), ("primary_mean", C.c_double),
                ("secondary_mean", C.c_double), ("correlation_coef", C.c_double)]


_HPGL_COK_M1_PARAMS = __hpgl_cockriging_m1_params_t
_HPGL_COK_M2_PARAMS = __hpgl_cockriging_m2_params_t


class _HPGL_SGS_PARAMS(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("kriging_kind", C.c_int), ("seed", C.c_long),
                ("min_neighbours", C.c_int)]


class hpgl_non_parametric_cdf_t(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_float)), ("probs", C.POINTER(C.c_float)), ("size", C.c_longlong)]


_HPGL_NON_PARAMETRIC_CDF = hpgl_non_parametric_cdf_t


class _HPGL_B200_OPTIONS(C.Structure):
    _fields_ = [("precision", C.c_int), ("refine_steps", C.c_int), ("flags", C.c_uint),
                ("stream", C.c_void_p), ("estimate64", C.c_void_p), ("variance", C.c_void_p),
                ("status", C.c_void_p), ("ik_probs", C.c_void_p), ("tolerance", C.c_double)]


FP64_PLAIN = 0
FP32_REFINED = 1
FLAG_DEVICE_POINTERS = 1
FLAG_OUT_IS_CLONE = 2
FLAG_EXACT_SEARCH = 4

LIB_NAME = "libhpgl_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

# Status codes of the _ex / b200 entry points (include/hpgl_b200.h)
OK, EINVAL, ECUDA, ENOMEM, ELIMIT = 0, -1, -2, -3, -4

# Exported symbols of include/hpgl_b200.h (checked by the test suite).
EXPORTS = [
    "hpgl_get_last_exception_message", "hpgl_set_output_handler", "hpgl_set_progress_handler",
    "hpgl_set_thread_num", "hpgl_get_thread_num", "hpgl_ordinary_kriging", "hpgl_simple_kriging",
    "hpgl_simple_kriging_weights", "hpgl_indicator_kriging", "hpgl_median_ik", "hpgl_lvm_kriging",
    "hpgl_sgs_simulation", "hpgl_sgs_lvm_simulation", "hpgl_simple_cokriging_mark1", "hpgl_simple_cokriging_mark2",
    "hpgl_b200_cokriging_ex", "hpgl_sis_simulation", "hpgl_sis_simulation_lvm", "hpgl_b200_sis_ex",
    "hpgl_b200_sim_levels",
    "hpgl_read_inc_file_float", "hpgl_read_inc_file_byte", "hpgl_write_inc_file_float",
    "hpgl_write_inc_file_byte", "hpgl_write_gslib_cont_property", "hpgl_write_gslib_byte_property",
    "hpgl_b200_cont_kriging_ex", "hpgl_b200_lvm_kriging_ex", "hpgl_b200_sgs_ex", "hpgl_b200_sgs_draws", "hpgl_b200_indicator_kriging_ex", "hpgl_b200_median_ik_ex",
    "hpgl_b200_find_neighbours", "hpgl_b200_last_stats", "hpgl_b200_host_alloc", "hpgl_b200_host_free",
    "hpgl_b200_transform", "hpgl_b200_template", "hpgl_b200_covariance", "hpgl_b200_version",
    "hpgl_b200_sk_weights_noalloc", "hpgl_b200_loo_ok", "hpgl_b200_loo_ok_adjoint",
    "hpgl_b200_solve_variant", "hpgl_b200_solve_variant_get", "hpgl_b200_tune_mode", "hpgl_b200_tune_load",
    "hpgl_b200_tune_save", "hpgl_b200_tune_reset",
]


def _load():
    if not os.path.isfile(LIB_PATH):
        raise ImportError(
            f"{LIB_NAME} is not built (expected at {LIB_PATH}); run `make -C hpgl-reborn_b200` "
            "or __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    _f32 = ndpointer(dtype="float32", flags="C")
    _u8 = ndpointer(dtype="uint8", flags="C")
    _f32F = ndpointer(dtype="float32", flags=("F", "W", "A"))
    _u8F = ndpointer(dtype="uint8", flags=("F", "W", "A"))
    i_p = C.POINTER(C.c_int)
    lib.hpgl_get_last_exception_message.restype = C.c_char_p
    lib.hpgl_get_last_exception_message.argtypes = []
    lib.hpgl_set_output_handler.restype = None
    lib.hpgl_set_output_handler.argtypes = [hpgl_output_handler, C.py_object]
    lib.hpgl_set_progress_handler.restype = None
    lib.hpgl_set_progress_handler.argtypes = [hpgl_progress_handler, C.py_object]
    lib.hpgl_set_thread_num.restype = None
    lib.hpgl_set_thread_num.argtypes = [C.c_int]
    lib.hpgl_get_thread_num.restype = C.c_int
    lib.hpgl_ordinary_kriging.restype = None
    lib.hpgl_ordinary_kriging.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_OK_PARAMS),
                                          C.POINTER(_HPGL_CONT_MASKED_ARRAY)]
    lib.hpgl_simple_kriging.restype = None
    lib.hpgl_simple_kriging.argtypes = [_f32F, _u8F, C.POINTER(_HPGL_SHAPE), C.POINTER(_HPGL_SK_PARAMS),
                                        _f32F, _u8F, C.POINTER(_HPGL_SHAPE)]
    lib.hpgl_simple_kriging_weights.restype = C.c_int
    lib.hpgl_simple_kriging_weights.argtypes = [C.POINTER(C.c_float), _f32, _f32, _f32, C.c_int,
                                                C.POINTER(_HPGL_COV_PARAMS), _f32]
    lib.hpgl_indicator_kriging.restype = None
    lib.hpgl_indicator_kriging.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.POINTER(_HPGL_IND_MASKED_ARRAY),
                                           C.POINTER(_HPGL_IK_PARAMS), C.c_int]
    lib.hpgl_median_ik.restype = None
    lib.hpgl_median_ik.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.POINTER(_HPGL_MEDIAN_IK_PARAMS),
                                   C.POINTER(_HPGL_IND_MASKED_ARRAY)]
    vp = C.c_void_p
    lib.hpgl_b200_cont_kriging_ex.restype = C.c_int
    lib.hpgl_b200_cont_kriging_ex.argtypes = [C.c_int, i_p, vp, vp, C.POINTER(_HPGL_SK_PARAMS), vp, vp,
                                              C.POINTER(_HPGL_B200_OPTIONS)]
    lib.hpgl_lvm_kriging.restype = None
    lib.hpgl_lvm_kriging.argtypes = [_f32F, _u8F, C.POINTER(_HPGL_SHAPE), _f32F, C.POINTER(_HPGL_SHAPE),
                                     C.POINTER(_HPGL_OK_PARAMS), _f32F, _u8F, C.POINTER(_HPGL_SHAPE)]
    lib.hpgl_b200_lvm_kriging_ex.restype = C.c_int
    lib.hpgl_b200_lvm_kriging_ex.argtypes = [i_p, vp, vp, vp, C.POINTER(_HPGL_OK_PARAMS), vp, vp,
                                             C.POINTER(_HPGL_B200_OPTIONS)]
    lib.hpgl_sgs_simulation.restype = None
    lib.hpgl_sgs_simulation.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_SGS_PARAMS),
                                        C.POINTER(_HPGL_NON_PARAMETRIC_CDF), C.POINTER(C.c_double),
                                        C.POINTER(_HPGL_UBYTE_ARRAY)]
    lib.hpgl_sgs_lvm_simulation.restype = None
    lib.hpgl_sgs_lvm_simulation.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_SGS_PARAMS),
                                            C.POINTER(_HPGL_NON_PARAMETRIC_CDF), C.POINTER(_HPGL_FLOAT_ARRAY),
                                            C.POINTER(_HPGL_UBYTE_ARRAY)]
    lib.hpgl_b200_sgs_ex.restype = C.c_int
    lib.hpgl_b200_sgs_ex.argtypes = [i_p, vp, vp, vp, C.POINTER(_HPGL_NON_PARAMETRIC_CDF), vp,
                                     C.POINTER(_HPGL_SGS_PARAMS), C.POINTER(_HPGL_B200_OPTIONS)]
    cma = C.POINTER(_HPGL_CONT_MASKED_ARRAY)
    lib.hpgl_simple_cokriging_mark1.restype = None
    lib.hpgl_simple_cokriging_mark1.argtypes = [cma, cma, C.POINTER(_HPGL_COK_M1_PARAMS), cma]
    lib.hpgl_simple_cokriging_mark2.restype = None
    lib.hpgl_simple_cokriging_mark2.argtypes = [cma, cma, C.POINTER(_HPGL_COK_M2_PARAMS), cma]
    lib.hpgl_b200_cokriging_ex.restype = C.c_int
    lib.hpgl_b200_cokriging_ex.argtypes = [C.c_int, i_p, vp, vp, vp, vp, C.POINTER(_HPGL_COK_M1_PARAMS),
                                           C.POINTER(_HPGL_COK_M2_PARAMS), vp, vp, C.POINTER(_HPGL_B200_OPTIONS)]
    lib.hpgl_read_inc_file_float.restype = C.c_int
    lib.hpgl_read_inc_file_float.argtypes = [C.c_char_p, C.c_float, C.c_int, _f32F, _u8F]
    lib.hpgl_read_inc_file_byte.restype = C.c_int
    lib.hpgl_read_inc_file_byte.argtypes = [C.c_char_p, C.c_int, C.c_int, _u8F, _u8F, _u8, C.c_int]
    lib.hpgl_write_inc_file_float.restype = C.c_int
    lib.hpgl_write_inc_file_float.argtypes = [C.c_char_p, C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.c_float, C.c_char_p]
    lib.hpgl_write_inc_file_byte.restype = C.c_int
    lib.hpgl_write_inc_file_byte.argtypes = [C.c_char_p, C.POINTER(_HPGL_IND_MASKED_ARRAY), C.c_int, C.c_char_p,
                                             C.POINTER(C.c_ubyte), C.c_int]
    lib.hpgl_write_gslib_cont_property.restype = C.c_int
    lib.hpgl_write_gslib_cont_property.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.c_char_p, C.c_char_p,
                                                   C.c_double]
    lib.hpgl_write_gslib_byte_property.restype = C.c_int
    lib.hpgl_write_gslib_byte_property.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.c_char_p, C.c_char_p,
                                                   C.c_double, C.POINTER(C.c_ubyte), C.c_int]
    ima = C.POINTER(_HPGL_IND_MASKED_ARRAY)
    lib.hpgl_sis_simulation.restype = None
    lib.hpgl_sis_simulation.argtypes = [ima, C.POINTER(_HPGL_IK_PARAMS), C.c_int, C.c_int, C.POINTER(_HPGL_UBYTE_ARRAY)]
    lib.hpgl_sis_simulation_lvm.restype = None
    lib.hpgl_sis_simulation_lvm.argtypes = [ima, C.POINTER(_HPGL_IK_PARAMS), C.POINTER(_HPGL_FLOAT_ARRAY), C.c_int,
                                            C.c_int, C.POINTER(_HPGL_UBYTE_ARRAY), C.c_int]
    lib.hpgl_b200_sis_ex.restype = C.c_int
    lib.hpgl_b200_sis_ex.argtypes = [i_p, vp, vp, vp, C.POINTER(_HPGL_IK_PARAMS), C.c_int, vp, C.c_int, C.c_int,
                                     C.POINTER(_HPGL_B200_OPTIONS)]
    lib.hpgl_b200_sim_levels.restype = C.c_int
    lib.hpgl_b200_sim_levels.argtypes = [C.c_longlong, C.c_int, vp, vp]
    lib.hpgl_b200_sgs_draws.restype = C.c_int
    lib.hpgl_b200_sgs_draws.argtypes = [C.c_longlong, C.c_longlong, vp]
    lib.hpgl_b200_indicator_kriging_ex.restype = C.c_int
    lib.hpgl_b200_indicator_kriging_ex.argtypes = [i_p, vp, vp, C.POINTER(_HPGL_IK_PARAMS), C.c_int, vp, vp,
                                                   C.POINTER(_HPGL_B200_OPTIONS)]
    lib.hpgl_b200_median_ik_ex.restype = C.c_int
    lib.hpgl_b200_median_ik_ex.argtypes = [i_p, vp, vp, C.POINTER(_HPGL_MEDIAN_IK_PARAMS), vp, vp,
                                           C.POINTER(_HPGL_B200_OPTIONS)]
    lib.hpgl_b200_find_neighbours.restype = C.c_int
    lib.hpgl_b200_find_neighbours.argtypes = [C.c_int, i_p, vp, C.POINTER(_HPGL_SK_PARAMS), vp, C.c_int, vp, vp,
                                              vp]
    lib.hpgl_b200_last_stats.restype = C.c_int
    lib.hpgl_b200_last_stats.argtypes = [C.POINTER(C.c_double), C.c_int]
    lib.hpgl_b200_solve_variant.restype = C.c_int
    lib.hpgl_b200_solve_variant.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    lib.hpgl_b200_solve_variant_get.restype = C.c_int
    lib.hpgl_b200_solve_variant_get.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.hpgl_b200_tune_mode.restype = C.c_int
    lib.hpgl_b200_tune_mode.argtypes = [C.c_int]
    lib.hpgl_b200_tune_load.restype = C.c_int
    lib.hpgl_b200_tune_load.argtypes = [C.c_char_p]
    lib.hpgl_b200_tune_save.restype = C.c_int
    lib.hpgl_b200_tune_save.argtypes = [C.c_char_p]
    lib.hpgl_b200_tune_reset.restype = None
    lib.hpgl_b200_tune_reset.argtypes = []
    lib.hpgl_b200_host_alloc.restype = C.c_void_p
    lib.hpgl_b200_host_alloc.argtypes = [C.c_size_t]
    lib.hpgl_b200_host_free.restype = None
    lib.hpgl_b200_host_free.argtypes = [C.c_void_p]
    lib.hpgl_b200_transform.restype = C.c_int
    lib.hpgl_b200_transform.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.hpgl_b200_template.restype = C.c_int
    lib.hpgl_b200_template.argtypes = [C.c_int, C.POINTER(_HPGL_COV_PARAMS), i_p, vp, C.c_int, i_p]
    lib.hpgl_b200_covariance.restype = C.c_double
    lib.hpgl_b200_covariance.argtypes = [C.c_int, C.POINTER(_HPGL_COV_PARAMS), i_p, i_p, i_p]
    lib.hpgl_b200_version.restype = C.c_char_p
    lib.hpgl_b200_sk_weights_noalloc.restype = C.c_int
    lib.hpgl_b200_sk_weights_noalloc.argtypes = [C.POINTER(C.c_float), _f32, _f32, _f32, C.c_int,
                                                 C.POINTER(_HPGL_COV_PARAMS), _f32, C.c_void_p]
    vp = C.c_void_p
    d9 = C.POINTER(C.c_double)
    loo_common = [vp, vp, C.c_int, vp, vp, vp, C.c_int, C.c_int, C.c_int, d9, C.c_double, C.c_double, C.c_double]
    lib.hpgl_b200_loo_ok.restype = C.c_int
    lib.hpgl_b200_loo_ok.argtypes = loo_common + [vp, vp, vp]
    lib.hpgl_b200_loo_ok_adjoint.restype = C.c_int
    lib.hpgl_b200_loo_ok_adjoint.argtypes = loo_common + [vp, vp, vp, vp]
    return lib


_hpgl_so = _load()


def last_error() -> str:
    msg = _hpgl_so.hpgl_get_last_exception_message()
    return msg.decode("utf-8", errors="replace") if msg else ""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc}): {last_error()}")


STATS_KEYS = (["total_ms", "search_ms", "solve_ms", "tie_cells", "template_cells", "kriged_cells",
               "kernel_launches", "h2d_bytes", "d2h_bytes", "escalated_cells", "search_kernel_ms"]
              + [f"bucket_items_{i}" for i in range(5)] + [f"bucket_ms_{i}" for i in range(5)]
              + [f"bucket_flops_{i}" for i in range(5)]
              + ["stage_" + s + "_ms" for s in ("upload", "compact", "tables", "bins", "search", "ties", "prepare",
                                              "solve", "finalize", "download")]
              + ["prefilter_exact_cells", "prefilter_active", "plan_ms", "sgs_levels", "sgs_draws_ms",
                 "sgs_flops", "refined_cells"])


VARIANT_DEFAULT, VARIANT_FOLD, VARIANT_QUAD, VARIANT_FOLD_NARROW, VARIANT_QUAD_NARROW, VARIANT_TILE = 0, 1, 2, 3, 4, 5
VARIANT_TILE_NARROW, VARIANT_WIDE = 6, 7
VARIANT_NAMES = {VARIANT_DEFAULT: "default", VARIANT_FOLD: "fold", VARIANT_QUAD: "quad",
                 VARIANT_FOLD_NARROW: "fold_narrow", VARIANT_QUAD_NARROW: "quad_narrow", VARIANT_TILE: "tile",
                 VARIANT_TILE_NARROW: "tile_narrow", VARIANT_WIDE: "wide"}


def solve_variant(bucket_np: int, cov_type: int, precision: int, variant: int = None) -> int:
    """The solve-kernel variant of one (bucket, covariance type, precision) key
    (hpgl_b200_solve_variant_get); with `variant`, set it and return the
    previous setting (hpgl_b200_solve_variant)."""
    if variant is None:
        return int(_hpgl_so.hpgl_b200_solve_variant_get(bucket_np, cov_type, precision))
    prev = int(_hpgl_so.hpgl_b200_solve_variant(bucket_np, cov_type, precision, variant))
    if prev < 0:
        raise ValueError(f"invalid solve variant {variant} for bucket {bucket_np}, cov type {cov_type}, "
                         f"precision {precision}")
    return prev


def last_stats() -> dict:
    """Timing and counters of the last engine call (hpgl_b200_last_stats)."""
    buf = (C.c_double * len(STATS_KEYS))()
    n = _hpgl_so.hpgl_b200_last_stats(buf, len(STATS_KEYS))
    return {k: float(buf[i]) for i, k in enumerate(STATS_KEYS[:n])}
