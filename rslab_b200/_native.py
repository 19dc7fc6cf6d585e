"""ctypes binding of librslab_b200.so (the C ABI in include/rslab_b200.h).

The library is required: importing this module raises if it is missing or does
not export every declared entry point.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librslab_b200.so"

F64, C64, F32, C32 = 0, 1, 2, 3
ORDER_AMD, ORDER_METIS_ND, ORDER_NATURAL, ORDER_GIVEN = 0, 1, 2, 3
PIVOT_FAIL, PIVOT_PERTURB, PIVOT_FORCE_ACCEPT = 0, 1, 2
SCALING_ONEPASS, SCALING_IDENTITY = 0, 1
SCHUR_TENSOR, SCHUR_FMA, SCHUR_AUTO = 0, 1, 2
METHOD_LEFT_LOOKING, METHOD_MULTIFRONTAL = 0, 1
TIER_FP64, TIER_FP32, TIER_TF32X3 = 0, 1, 2
TIER_MLP_PARAMS = 4931

i64p = C.POINTER(C.c_int64)
i32p = C.POINTER(C.c_int32)
fp = C.POINTER(C.c_float)
vp = C.c_void_p


class AnalyzeSettings(C.Structure):
    _fields_ = [
        ("ordering", C.c_int32),
        ("nemin", C.c_int64),
        ("relax", C.c_int32),
        ("relax_max_width", C.c_int64),
        ("relax_max_extra_rows", C.c_int64),
        ("hybrid_liu", C.c_int32),
        ("panel_nb", C.c_int64),
        ("given_perm", i64p),
    ]


class FactorSettings(C.Structure):
    _fields_ = [
        ("on_zero_pivot", C.c_int32),
        ("abs_floor", C.c_double),
        ("scaling", C.c_int32),
        ("use_graph", C.c_int32),
        ("stream", vp),
        ("schur_engine", C.c_int32),
        ("drop_tol", C.c_double),
        ("overlap", C.c_int32),
        ("method", C.c_int32),
    ]


class SymbolicInfo(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("nnz", C.c_int64), ("nsuper", C.c_int64), ("nlevels", C.c_int64),
        ("factor_nnz_sym", C.c_int64), ("panel_elems", C.c_int64),
        ("flops_model", C.c_double), ("flops_proxy", C.c_double),
        ("renumbered", C.c_int32),
        ("amd_ncmpa", C.c_int64), ("amd_ndense", C.c_int64),
        ("amd_ndiv", C.c_double), ("amd_nms_ldl", C.c_double), ("amd_nms_lu", C.c_double),
        ("n_factor_launches", C.c_int64), ("n_solve_launches", C.c_int64),
        ("tc_tiles", C.c_int64), ("tc_pairs", C.c_int64), ("tc_chunks_complex", C.c_int64),
        ("tc_chunks_real", C.c_int64),
    ]


class FactorInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("failing_supernode", C.c_int64),
        ("inertia_pos", C.c_int64), ("inertia_neg", C.c_int64), ("inertia_zero", C.c_int64),
        ("n_perturbed", C.c_int64), ("factor_ms", C.c_double), ("solve_ms", C.c_double),
        ("dtype", C.c_int32), ("dtype_hi", C.c_int32), ("multiprocessors", C.c_int32),
        ("schur_engine", C.c_int32), ("method", C.c_int32),
    ]


class MemoryEstimateC(C.Structure):
    _fields_ = [
        ("value_bytes", C.c_int64), ("factor_nnz", C.c_int64), ("factor_bytes", C.c_int64),
        ("panels_all_bytes", C.c_int64), ("panel_live_peak_bytes", C.c_int64), ("transient_peak_bytes", C.c_int64),
        ("factor_flops", C.c_uint64), ("critical_path_flops", C.c_uint64), ("max_tree_width", C.c_int64),
        ("symbolic_factor_nnz", C.c_int64), ("mf_transient_peak_bytes", C.c_int64),
    ]


class MixedInfoC(C.Structure):
    _fields_ = [
        ("ir_iters", C.c_int64), ("gmres_iters", C.c_int64),
        ("backward_error", C.c_double), ("certified", C.c_int32),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "rslab_version": (C.c_int, []),
    "rslab_last_error": (C.c_char_p, []),
    "rslab_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "rslab_default_analyze_settings": (None, [C.POINTER(AnalyzeSettings)]),
    "rslab_default_factor_settings": (None, [C.POINTER(FactorSettings)]),
    "rslab_analyze": (C.c_int, [C.c_int64, i64p, i64p, C.POINTER(AnalyzeSettings), C.POINTER(vp)]),
    "rslab_analyze_tuned": (C.c_int, [C.c_int64, i64p, i64p, C.c_int64, C.POINTER(vp), C.POINTER(C.c_int32)]),
    "rslab_symbolic_estimate": (C.c_int, [vp, C.c_int64, C.POINTER(MemoryEstimateC)]),
    "rslab_validate_lower_csc": (C.c_int, [C.c_int64, i64p, i64p, C.c_int64]),
    "rslab_symbolic_info": (C.c_int, [vp, C.POINTER(SymbolicInfo)]),
    "rslab_symbolic_export": (C.c_int, [vp, i64p, i64p, i64p, i64p, i64p, i64p, i64p, i64p, i64p]),
    "rslab_free_symbolic": (None, [vp]),
    "rslab_factor": (C.c_int, [vp, C.c_int, vp, C.c_int, C.POINTER(FactorSettings), C.POINTER(vp)]),
    "rslab_refactor": (C.c_int, [vp, vp, C.c_int]),
    "rslab_solve": (C.c_int, [vp, vp, C.c_int64, vp, C.c_int]),
    "rslab_set_pivot_reuse": (C.c_int, [vp, C.c_int]),
    "rslab_factor_info": (C.c_int, [vp, C.POINTER(FactorInfo)]),
    "rslab_factor_stream": (vp, [vp]),
    "rslab_export_factors": (C.c_int, [vp, i64p, i64p, vp, vp, vp, C.POINTER(C.c_uint8), i64p,
                                       C.POINTER(C.c_double), i64p]),
    "rslab_factor_profile": (C.c_int, [vp, C.POINTER(C.c_double), i64p, C.POINTER(C.c_double)]),
    "rslab_solve_profile": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_double), i64p]),
    "rslab_analyze_batch": (C.c_int, [C.c_int64, i64p, C.POINTER(i64p), C.POINTER(i64p),
                                      C.POINTER(AnalyzeSettings), C.POINTER(vp)]),
    "rslab_batch_layout": (C.c_int, [vp, i64p, i64p, i64p]),
    "rslab_mixed_batch_result": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_double), i64p]),
    "rslab_solve_refined": (C.c_int, [vp, vp, C.c_int64, C.c_int64, vp, C.c_int]),
    "rslab_profile_trace": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_float), i64p]),
    "rslab_free_factor": (None, [vp]),
    "rslab_mixed_factor": (C.c_int, [vp, C.c_int, vp, C.c_int, C.POINTER(FactorSettings), C.POINTER(vp)]),
    "rslab_mixed_solve": (C.c_int, [vp, vp, C.c_int64, C.c_double, vp, C.c_int, C.POINTER(MixedInfoC)]),
    "rslab_gmres_block": (C.c_int, [vp, vp, C.c_int64, C.c_double, C.c_int64, C.c_int64, vp, vp, C.c_int, i64p,
                                    C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "rslab_tier_factor": (C.c_int, [vp, C.c_int, C.c_int, vp, C.c_int, C.POINTER(FactorSettings), C.POINTER(vp)]),
    "rslab_tier_mlp_forward": (C.c_int, [fp, fp, C.c_int64, fp, C.c_int]),
    "rslab_tier_mlp_grad": (C.c_int, [fp, fp, i32p, fp, C.c_int64, fp, fp, C.c_int]),
    "rslab_tier_mlp_train": (C.c_int, [fp, fp, i32p, fp, C.c_int64, C.c_int64, C.c_float, fp, C.c_int]),
    "rslab_rng_units": (C.c_uint64, [C.c_uint64, C.c_int64, C.POINTER(C.c_double)]),
    "rslab_amd_order": (C.c_int, [C.c_int64, i64p, i64p, i64p, C.POINTER(C.c_double)]),
    "rslab_metis_order": (C.c_int, [C.c_int64, i64p, i64p, C.c_uint64, C.c_int, C.c_int64, i64p]),
    "rslab_compress_factors": (C.c_int, [vp, C.POINTER(vp)]),
    "rslab_cfac_info": (C.c_int, [vp, i64p, i64p, i64p, i32p]),
    "rslab_cfac_export": (C.c_int, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), vp, vp, vp,
                                    C.POINTER(C.c_uint8), C.POINTER(C.c_uint32)]),
    "rslab_cfac_solve": (C.c_int, [vp, vp, vp]),
    "rslab_free_cfac": (None, [vp]),
    "rslab_panel_factor_noalloc": (C.c_int, [C.c_int, vp, C.c_int64, C.c_int64, C.c_int64, vp, vp, vp, vp, vp,
                                             vp]),
}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python rslab_b200/build.py` "
            "(there is no CPU fallback for the LDL^T path)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if the export is missing
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    msg = lib.rslab_last_error()
    return msg.decode() if msg else ""
