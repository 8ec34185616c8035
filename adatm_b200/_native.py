"""ctypes declarations of libadatm_b200.so (include/splatt.h, include/adatm_b200.h).

The library must exist in-tree (``python -m adatm_b200.build`` or
``__graft_entry__.build()``); when it is missing and nvcc is on the machine it
is built on first use. There is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_NMODES = 88

SPLATT_SUCCESS = 1
SPLATT_ERROR_BADINPUT = 2
SPLATT_ERROR_NOMEMORY = 3
ADATM_ERROR_CUDA = 4

u64 = C.c_uint64
P_u64 = C.POINTER(u64)
P_f64 = C.POINTER(C.c_double)


class CsfSparsity(C.Structure):
    _fields_ = [("nfibs", u64 * MAX_NMODES), ("fptr", P_u64 * MAX_NMODES),
                ("fids", P_u64 * MAX_NMODES), ("vals", P_f64)]


class SplattCsf(C.Structure):
    _fields_ = [("nnz", u64), ("nmodes", u64), ("dims", u64 * MAX_NMODES),
                ("dim_perm", u64 * MAX_NMODES), ("which_tile", C.c_int), ("ntiles", u64),
                ("tile_dims", u64 * MAX_NMODES), ("pt", C.POINTER(CsfSparsity))]


class SplattKruskal(C.Structure):
    _fields_ = [("rank", u64), ("factors", P_f64 * MAX_NMODES), ("lambda_", P_f64),
                ("nmodes", u64), ("dims", u64 * MAX_NMODES), ("fit", C.c_double)]


class RcsfSeq(C.Structure):
    _fields_ = [("begin_imten", u64), ("n_imten", u64), ("rcsfs", C.POINTER(SplattCsf))]


class GroupProperties(C.Structure):
    _fields_ = [("memo_mode", u64), ("begin_imten", u64), ("n_imten", u64), ("o_opt", P_u64)]


class MatrixT(C.Structure):
    _fields_ = [("I", u64), ("J", u64), ("vals", P_f64), ("rowmajor", C.c_int)]


class SpTensorT(C.Structure):
    _fields_ = [("nnz", u64), ("nmodes", u64), ("dims", P_u64), ("ind", C.POINTER(P_u64)),
                ("vals", P_f64), ("tiled", C.c_int), ("type", C.c_int)]


class AdatmPlan(C.Structure):
    _fields_ = [("nmodes", C.c_int), ("n_grp", C.c_int), ("memo_mode", u64 * 8),
                ("begin_imten", u64 * 8), ("n_imten", u64 * 8), ("o_opt", (u64 * 8) * 8),
                ("use_csfs", u64 * 8), ("use_tags", u64 * 8), ("space_efficient", C.c_int)]


class AdatmCandidate(C.Structure):
    _fields_ = [("plan", AdatmPlan), ("pspace", u64), ("pops", u64)]


def library_path() -> str:
    return os.path.join(HERE, "libadatm_b200.so")


_lib = None
_lock = threading.Lock()


def build(force: bool = False) -> str:
    from .build import build as _b
    return _b(force=force)


# (name, restype, argtypes)
_SIGS = [
    ("splatt_default_opts", P_f64, []),
    ("splatt_free_opts", None, [P_f64]),
    ("splatt_csf_convert", C.c_int, [u64, u64, C.POINTER(P_u64), P_f64,
                                     C.POINTER(C.POINTER(SplattCsf)), P_f64]),
    ("splatt_csf_load", C.c_int, [C.c_char_p, P_u64, C.POINTER(C.POINTER(SplattCsf)), P_f64]),
    ("splatt_free_csf", None, [C.POINTER(SplattCsf), P_f64]),
    ("splatt_free_kruskal", None, [C.POINTER(SplattKruskal)]),
    ("splatt_cpd_als", C.c_int, [C.POINTER(SplattCsf), u64, P_f64, C.POINTER(SplattKruskal)]),
    ("splatt_mttkrp", C.c_int, [u64, u64, C.POINTER(SplattCsf), C.POINTER(P_f64), P_f64, P_f64]),
    ("decide_product_order", None, [C.POINTER(SpTensorT), C.POINTER(P_u64)]),
    ("decide_parameters_auto", u64, [C.POINTER(SpTensorT), u64, C.c_int, C.POINTER(P_u64),
                                     C.POINTER(C.POINTER(GroupProperties))]),
    ("decide_candidate_configs", u64, [C.POINTER(SpTensorT), C.POINTER(P_u64), C.c_void_p]),
    ("csf_alloc_adaptive", C.POINTER(SplattCsf), [C.POINTER(SpTensorT), C.POINTER(GroupProperties),
                                                   u64, P_f64, P_u64]),
    ("rcsf_alloc_adaptive", C.POINTER(RcsfSeq), [C.POINTER(SplattCsf), u64, C.POINTER(GroupProperties),
                                                  u64, u64, P_f64, P_u64]),
    ("csf_storage_adaptive", C.c_size_t, [C.POINTER(SplattCsf), u64, C.POINTER(GroupProperties), C.c_int]),
    ("rcsf_storage_adaptive", C.c_size_t, [C.POINTER(RcsfSeq), u64]),
    ("decide_use_csfs", None, [u64, C.POINTER(GroupProperties), C.c_int, u64, P_u64, P_u64]),
    ("mttkrp_csf_adaptive", None, [C.POINTER(SplattCsf), C.POINTER(RcsfSeq), u64,
                                   C.POINTER(C.POINTER(MatrixT)), u64, C.c_void_p,
                                   C.POINTER(GroupProperties), C.c_int, u64, u64, P_f64]),
    ("cpd_als_iterate_adaptive", C.c_double, [C.POINTER(SplattCsf), C.POINTER(RcsfSeq), u64,
                                              C.POINTER(GroupProperties), u64, P_u64, P_u64,
                                              C.POINTER(C.POINTER(MatrixT)), P_f64, u64,
                                              C.c_void_p, P_f64]),
    ("splatt_cpd_als_adaptive", C.c_int, [C.POINTER(SplattCsf), C.POINTER(RcsfSeq), u64,
                                          C.POINTER(GroupProperties), u64, P_u64, P_u64, u64,
                                          P_f64, C.POINTER(SplattKruskal)]),
    ("bench_adaptm", None, [C.POINTER(SpTensorT), C.POINTER(C.POINTER(MatrixT)), C.c_void_p]),
    ("adatm_rcsf_pull", C.c_int, [C.POINTER(RcsfSeq), u64]),
    ("adatm_csf_tree_count", C.c_int, [C.POINTER(SplattCsf), C.POINTER(C.c_int)]),
    ("adatm_free_groups", None, [C.POINTER(GroupProperties), u64]),
    ("adatm_last_error", C.c_char_p, []),
    ("adatm_set_device", C.c_int, [C.c_int]),
    ("adatm_tensor_from_coo", C.c_int, [C.c_int, u64, P_u64, C.POINTER(P_u64), P_f64, C.c_int,
                                        C.POINTER(C.c_void_p)]),
    ("adatm_tensor_generate", C.c_int, [C.c_int, P_u64, u64, P_f64, C.c_int, C.c_double,
                                        C.c_double, u64, C.POINTER(C.c_void_p)]),
    ("adatm_tensor_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), P_u64, P_u64]),
    ("adatm_tensor_download", C.c_int, [C.c_void_p, P_u64, P_f64]),
    ("adatm_tensor_free", None, [C.c_void_p]),
    ("adatm_tensor_count_nfibs", C.c_int, [C.c_void_p, P_u64, P_u64]),
    ("adatm_plan_analytic", C.c_int, [C.c_void_p, u64, C.c_int, C.POINTER(AdatmPlan),
                                      C.POINTER(AdatmCandidate), C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
    ("adatm_plan_splatt", C.c_int, [C.c_void_p, C.c_int, C.POINTER(AdatmPlan)]),
    ("adatm_engine_create", C.c_int, [C.c_void_p, u64, C.POINTER(AdatmPlan), C.c_int, C.c_uint32,
                                      C.c_uint32, C.POINTER(C.c_void_p)]),
    ("adatm_engine_free", None, [C.c_void_p]),
    ("adatm_engine_csf_count", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("adatm_engine_csf_shape", C.c_int, [C.c_void_p, C.c_int, P_u64, P_u64]),
    ("adatm_engine_csf_arrays", C.c_int, [C.c_void_p, C.c_int, C.POINTER(P_u64), C.POINTER(P_u64), P_f64]),
    ("adatm_engine_memory", C.c_int, [C.c_void_p, P_u64, P_u64]),
    ("adatm_engine_init_factors", C.c_int, [C.c_void_p, u64]),
    ("adatm_engine_set_factors", C.c_int, [C.c_void_p, C.POINTER(P_f64)]),
    ("adatm_engine_get_factors", C.c_int, [C.c_void_p, C.POINTER(P_f64), P_f64]),
    ("adatm_engine_mttkrp", C.c_int, [C.c_void_p, u64, P_f64]),
    ("adatm_engine_mttkrp_direct", C.c_int, [C.c_void_p, u64, P_f64]),
    ("adatm_engine_memo", C.c_int, [C.c_void_p, C.c_int, C.c_int, P_f64]),
    ("adatm_engine_als", C.c_int, [C.c_void_p, u64, C.c_double, C.c_int, P_f64, P_u64, P_f64]),
    ("adatm_engine_als_begin", C.c_int, [C.c_void_p, C.c_int]),
    ("adatm_engine_time_sweeps", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    ("adatm_engine_time_mttkrp", C.c_int, [C.c_void_p, u64, C.c_int, C.POINTER(C.c_float)]),
    ("adatm_engine_fit", C.c_int, [C.c_void_p, P_f64]),
    ("adatm_engine_mttkrp_into", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("adatm_engine_update_from", C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    ("adatm_engine_fit_step", C.c_int, [C.c_void_p, P_f64]),
    ("adatm_engine_ttnorm", C.c_int, [C.c_void_p, P_f64]),
    ("adatm_engine_set_ttnorm", C.c_int, [C.c_void_p, C.c_double]),
    ("adatm_engine_mttkrp_bytes", C.c_int, [C.c_void_p, u64, P_f64]),
    ("adatm_engine_hot_rows", C.c_int, [C.c_void_p, u64, C.POINTER(C.c_int)]),
    ("adatm_engine_autotune", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.c_int, C.c_int, C.POINTER(C.c_int)]),
    ("adatm_engine_set_resident_grid", C.c_int, [C.c_void_p, C.c_int]),
    ("adatm_engine_set_walkers", C.c_int, [C.c_void_p, C.c_int]),
    ("adatm_engine_set_fold", C.c_int, [C.c_void_p, C.c_int]),
    ("adatm_engine_set_deterministic", C.c_int, [C.c_void_p, C.c_int]),
    ("adatm_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    ("adatm_batch_begin", C.c_int, [C.c_void_p]),
    ("adatm_batch_time_sweeps", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    ("adatm_batch_kernels", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("adatm_batch_free", None, [C.c_void_p]),
    ("adatm_plan_features", C.c_int, [C.c_void_p, u64, C.POINTER(C.c_float), P_f64,
                                      C.POINTER(AdatmCandidate), C.c_int, C.POINTER(C.c_int)]),
    ("adatm_mlp_create", C.c_int, [C.c_int, C.POINTER(C.c_int), u64, C.POINTER(C.c_void_p)]),
    ("adatm_mlp_free", None, [C.c_void_p]),
    ("adatm_mlp_nparams", C.c_int, [C.c_void_p, P_u64]),
    ("adatm_mlp_set_params", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("adatm_mlp_get_params", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("adatm_mlp_forward", C.c_int, [C.c_void_p, C.POINTER(C.c_float), u64, C.POINTER(C.c_float)]),
    ("adatm_mlp_gradient", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), u64,
                                     C.POINTER(C.c_float), P_f64]),
    ("adatm_mlp_train", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), u64,
                                  C.c_int, C.c_int, C.c_float, u64, P_f64]),
    ("adatm_plan_learned", C.c_int, [C.c_void_p, u64, C.c_void_p, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float), C.POINTER(AdatmPlan), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
    ("adatm_gram", C.c_int, [C.c_void_p, u64, C.c_int, C.c_int, C.c_void_p]),
    ("adatm_gram_noalloc", C.c_int, [C.c_void_p, u64, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    ("adatm_engine_launch_counts", C.c_int, [C.c_void_p, u64, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
]

EXPORTED = [name for name, _, _ in _SIGS]


def lib():
    """Load (building if absent) libadatm_b200.so and declare its prototypes."""
    global _lib
    with _lock:
        if _lib is None:
            path = library_path()
            if not os.path.exists(path):
                build()
            L = C.CDLL(path)
            for name, res, args in _SIGS:
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    if _lib is None:
        return ""
    s = _lib.adatm_last_error()
    return s.decode() if s else ""
