"""ctypes binding of libaifmm_b200.so (declared in include/aifmm_b200.h).

The library is loaded from rcs_b200/lib/ only; if it is missing the import
fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libaifmm_b200.so")

AIFMM_OK = 0
ERRORS = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ETIMEOUT", -5: "ESTATE", -6: "ESINGULAR", -7: "ENOTIMPL",
          -8: "EOVERFLOW"}

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_pp = C.POINTER(C.c_void_p)
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")

# name -> (restype, argtypes); every function returns an int status.
SIGNATURES = {
    "aifmm_last_error": (C.c_char_p, []),
    "aifmm_ctx_create": (_i, [_i, _pp]),
    "aifmm_ctx_destroy": (_i, [_p]),
    "aifmm_ctx_synchronize": (_i, [_p]),
    "aifmm_ctx_stream": (_i, [_p, _pp]),
    "aifmm_ctx_tune_report": (_i, [_p, C.c_char_p, _i, C.POINTER(_i)]),
    "aifmm_ctx_set_gemm_tiling": (_i, [_p, _i, _i]),
    "aifmm_ctx_memory": (_i, [_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "aifmm_ctx_trim": (_i, [_p]),
    "aifmm_kernel_create_efie": (_i, [_p, _dp, _i, _ip, _i, _d, _pp]),
    "aifmm_kernel_create_es": (_i, [_p, _dp, _i, _ip, _p, _i, _pp]),
    "aifmm_kernel_destroy": (_i, [_p]),
    "aifmm_kernel_set_plane_projection": (_i, [_p, _i]),
    "aifmm_kernel_size": (_i, [_p, C.POINTER(_i)]),
    "aifmm_kernel_locations": (_i, [_p, _dp]),
    "aifmm_kernel_matrix": (_i, [_p, _ip, _i, _ip, _i, _i, _p, _i]),
    "aifmm_kernel_matrix_device": (_i, [_p, _p, _i, _p, _i, _i, _p, _i]),
    "aifmm_kernel_rhs_reference": (_i, [_p, _dp, _dp]),
    "aifmm_kernel_rhs_plane": (_i, [_p, _dp, _dp, _dp]),
    "aifmm_kernel_rhs_conductor": (_i, [_p, _i, _dp]),
    "aifmm_kernel_currents": (_i, [_p, _dp, _dp]),
    "aifmm_kernel_rcs": (_i, [_p, _dp, _i, _dp, _dp, _dp]),
    "aifmm_solver_create": (_i, [_p, _p, _pp]),
    "aifmm_solver_create_at": (_i, [_p, _p, _dp, _i, _p, _pp]),
    "aifmm_solver_tree_order": (_i, [_p, _ip]),
    "aifmm_solver_factorize": (_i, [_p]),
    "aifmm_solver_solve": (_i, [_p, _dp, _i, _dp]),
    "aifmm_solver_set_graph_solve": (_i, [_p, _i]),
    "aifmm_solver_solve_device": (_i, [_p, _p, _i, _p]),
    "aifmm_solver_get_info": (_i, [_p, _p]),
    "aifmm_solver_destroy": (_i, [_p]),
    "aifmm_solver_checkpoint": (_i, [_p]),
    "aifmm_solver_rewind": (_i, [_p]),
    "aifmm_solver_save": (_i, [_p, C.c_char_p]),
    "aifmm_batch_factorize": (_i, [C.POINTER(_p), _i, _i, C.POINTER(_d)]),
    "aifmm_batch_solve_gmres": (_i, [C.POINTER(_p), C.POINTER(_p), C.POINTER(_p), C.POINTER(_i), C.POINTER(_p), _i,
                                     _d, _i, _i, _i, _p, C.POINTER(_d)]),
    "aifmm_solver_load": (_i, [_p, C.c_char_p, _pp]),
    "aifmm_launch_count": (_i, [C.POINTER(C.c_long)]),
    "aifmm_tc5_timeouts": (_i, [C.POINTER(C.c_long)]),
    "aifmm_debug_gemm_hold": (_i, [_p, _i]),
    "aifmm_mlp_num_params": (_i, [C.POINTER(_i)]),
    "aifmm_mlp_create": (_i, [_p, C.c_ulonglong, _pp]),
    "aifmm_mlp_destroy": (_i, [_p]),
    "aifmm_mlp_set_normalization": (_i, [_p, _fp, _fp]),
    "aifmm_mlp_get_params": (_i, [_p, _fp]),
    "aifmm_mlp_set_params": (_i, [_p, _fp]),
    "aifmm_mlp_infer": (_i, [_p, _fp, _i, _fp]),
    "aifmm_mlp_grad": (_i, [_p, _fp, _fp, _i, _fp, C.POINTER(C.c_float)]),
    "aifmm_mlp_train": (_i, [_p, _fp, _fp, _i, _i, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "aifmm_ctx_set_rank_model": (_i, [_p, _p, _d]),
    "aifmm_solver_aca_log": (_i, [_p, _p, _p, _p, _i, C.POINTER(_i)]),
    "aifmm_profile_ops": (_i, [_i]),
    "aifmm_profile_ops_read": (_i, [C.c_char_p, _i]),
    "aifmm_aca": (_i, [_p, _ip, _i, _ip, _i, _d, _ip, _ip, C.POINTER(_i), _dp, _dp]),
    "aifmm_rrqr": (_i, [_p, _dp, _i, _i, _i, _i, _i, _d, _i, _i, _dp, C.POINTER(_i), C.POINTER(_d)]),
    "aifmm_rrqr_full": (_i, [_p, _dp, _i, _i, _i, _i, _i, _d, _i, _i, _dp, _dp, _ip, C.POINTER(_i), C.POINTER(_d)]),
    "aifmm_rrqr_noalloc": (_i, [_p, _i, _i, _i, _i, _i, _d, _i, _i, _p, _p, _p, _p]),
    "aifmm_lu_solve": (_i, [_p, _dp, _i, _dp, _i, _dp]),
    "aifmm_zgemm": (_i, [_p, _i, _i, _i, _i, _i, _i, _dp, _dp, _i, _dp, _i, _dp, _dp, _i]),
    "aifmm_zgemm_device": (_i, [_p, _i, _i, _i, _i, _i, _i, _dp, _p, _i, _p, _i, _dp, _p, _i]),
    "aifmm_solver_dump": (_i, [_p, _p, C.c_long, C.POINTER(C.c_long)]),
    "aifmm_operator_create": (_i, [_p, _p, _pp]),
    "aifmm_operator_apply": (_i, [_p, _dp, _i, _dp]),
    "aifmm_operator_apply_device": (_i, [_p, _p, _i, _p]),
    "aifmm_operator_info": (_i, [_p, C.POINTER(_d), C.POINTER(_d)]),
    "aifmm_operator_destroy": (_i, [_p]),
    "aifmm_solver_solve_gmres": (_i, [_p, _p, _dp, _i, _dp, _d, _i, _i, _p]),
    "aifmm_solver_solve_gmres_device": (_i, [_p, _p, _p, _i, _p, _d, _i, _i, _p]),
    "aifmm_profile_gemm": (_i, [_i]),
    "aifmm_profile_gemm_read": (_i, [C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_long)]),
    "aifmm_profile_gemm_table": (_i, [C.c_char_p, _i]),
}


class SolverParams(C.Structure):
    _fields_ = [("leaf_size", C.c_int), ("tol_pow", C.c_int), ("fillin_tol", C.c_int), ("fillin_rank", C.c_int),
                ("n_levels", C.c_int), ("precision", C.c_int), ("exact_rrqr", C.c_int),
                ("drop_pow", C.c_int)]


class SolverInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("n_levels", C.c_int), ("start_level", C.c_int), ("avg_leaf_size", C.c_int),
                ("avg_multipoles", C.c_int), ("max_rank", C.c_int), ("n_rrqr", C.c_long),
                ("n_compress_p2p", C.c_long), ("n_compress_p2l", C.c_long), ("n_aca", C.c_long),
                ("n_aca_retry", C.c_long), ("kernels", C.c_long), ("t_assemble", C.c_double),
                ("t_factor", C.c_double), ("t_solve", C.c_double), ("flops_factor", C.c_double),
                ("mem_gb", C.c_double), ("mem_after_gb", C.c_double), ("t_rrqr", C.c_double),
                ("t_compress", C.c_double), ("t_elim_x", C.c_double), ("t_elim_z", C.c_double),
                ("t_nonleaf", C.c_double), ("t_lu", C.c_double), ("t_msolve", C.c_double),
                ("t_schur", C.c_double), ("t_aca", C.c_double), ("aca_ws_bytes", C.c_double),
                ("n_aca_launches", C.c_long), ("n_solve_graph", C.c_long), ("n_solve_capture", C.c_long)]

class GmresInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("cycles", C.c_int), ("relres", C.c_double), ("t_precond", C.c_double),
                ("t_matvec", C.c_double)]


_lib = None


class AifmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m rcs_b200.build` "
                              "(the CUDA library is required; there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != AIFMM_OK:
        raise AifmmError(rc, lib().aifmm_last_error().decode())


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
