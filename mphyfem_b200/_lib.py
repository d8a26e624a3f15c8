"""ctypes binding of libmphy.so (the C ABI declared in include/mphy.h).

The library is built in-tree by ``mphyfem_b200.build``. There is no fallback: if the shared
object is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmphy.so")

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)
_vp = C.c_void_p

# status codes (include/mphy.h)
OK = 0
ERR_INVALID_ARG = 1
ERR_CUDA = 2
ERR_NO_DEVICE = 3
ERR_OUT_OF_MEMORY = 4
ERR_UNSUPPORTED = 5
ERR_STATE = 6
ERR_NEG_JACOBIAN = 7
ERR_NOT_CONVERGED = 8
ERR_INDEFINITE = 9
ERR_DIVERGED = 10
ERR_TIME_STEP = 11

SOLVER_EMPTY, PATTERN_OK, INIT_OK, ASSEMBLY_OK, FACTORISE_OK = range(5)
PREC_FP64, PREC_MIXED, PREC_MIXED_F32VEC, PREC_MIXED_TC = 0, 1, 2, 3
PC_JACOBI, PC_FSAI, PC_FSAI_LEARNED = 0, 1, 2
TANGENT_REFERENCE, TANGENT_CONSISTENT = 0, 1
MAT_NEOHOOKEAN, MAT_MOONEYRIVLIN, MAT_GENT, MAT_ARRUDABOYCE = 0, 1, 2, 3
MAT_NDATA = 4


class SolverOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("pc_type", C.c_int32), ("tangent", C.c_int32), ("max_it", C.c_int32),
        ("rtol", C.c_double), ("abstol", C.c_double), ("dtol", C.c_double), ("inner_rtol", C.c_double),
        ("max_outer", C.c_int32), ("chunk", C.c_int32), ("coarse_aggregates", C.c_int32), ("norm_type", C.c_int32),
        ("coarse_modes", C.c_int32), ("coarse_lag", C.c_int32),
    ]


class NewtonOpts(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("t_final", C.c_double), ("max_steps", C.c_int32), ("max_newton", C.c_int32),
        ("tol_rel", C.c_double), ("tol_abs", C.c_double),
    ]


class IterStats(C.Structure):
    _fields_ = [
        ("step", C.c_int32), ("iter", C.c_int32), ("krylov_its", C.c_int32), ("status", C.c_int32),
        ("rhs_norm", C.c_double), ("t_assembly_ms", C.c_double), ("t_solve_ms", C.c_double),
        ("kernel_launches", C.c_int64),
    ]


class MixedOpts(C.Structure):
    _fields_ = [("tangent", C.c_int32), ("max_it", C.c_int32), ("rtol", C.c_double),
                ("coarse_aggregates", C.c_int32), ("coarse_modes", C.c_int32)]


class BatchStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int32), ("graph_replays", C.c_int32), ("kernel_launches", C.c_int64), ("t_ms", C.c_float),
    ]


class MphyError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"mphy status {status} ({status_string(status)}): {message}")
        self.status = status


# every exported symbol with (restype, argtypes); include/mphy.h is the source of truth
SIGNATURES = {
    "mphy_status_string": (C.c_char_p, [C.c_int]),
    "mphy_last_error": (C.c_char_p, []),
    "mphy_api_version": (C.c_int, []),
    "mphy_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "mphy_ctx_destroy": (C.c_int, [_vp]),
    "mphy_ctx_synchronize": (C.c_int, [_vp]),
    "mphy_ctx_stream": (_vp, [_vp]),
    "mphy_mesh_create": (C.c_int, [_vp, C.c_int32, _d, C.c_int32, C.c_int32, _i32, _i32, C.c_int32, _d, _u8,
                                   C.POINTER(_vp)]),
    "mphy_mesh_destroy": (C.c_int, [_vp]),
    "mphy_mesh_set_prescribed": (C.c_int, [_vp, _d, _d]),
    "mphy_material_nh_eval": (C.c_int, [_vp, C.c_int32, _vp, C.c_double, C.c_double, C.c_int32, C.c_int32, _vp, _vp]),
    "mphy_mesh_set_materials": (C.c_int, [_vp, C.c_int32, _i32, _d]),
    "mphy_material_eval": (C.c_int, [_vp, C.c_int32, _vp, C.c_int32, _d, C.c_double, C.c_int32, C.c_int32, _vp,
                                     _vp]),
    "mphy_elem_eval_tc": (C.c_int, [_vp, _vp, _vp, C.c_int32, _vp, _vp, _i64]),
    "mphy_elem_eval": (C.c_int, [_vp, _vp, _vp, C.c_int32, _vp, _vp, _i64]),
    "mphy_elem_eval_noalloc": (C.c_int, [_vp, C.c_int32, _vp, C.c_int32, C.c_int32, _vp, _vp, C.c_int32, _vp, _vp,
                                         C.c_int32, _vp, _vp, _i64]),
    "mphy_pattern_build": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "mphy_pattern_info": (C.c_int, [_vp, _i32, _i64, _i64, _i64]),
    "mphy_pattern_export_csr": (C.c_int, [_vp, _i64, _i32]),
    "mphy_pattern_export_dofmap": (C.c_int, [_vp, _i32, _i32]),
    "mphy_pattern_destroy": (C.c_int, [_vp]),
    "mphy_solver_opts_default": (None, [C.POINTER(SolverOpts)]),
    "mphy_solver_create": (C.c_int, [_vp, _vp, _vp, C.POINTER(SolverOpts), C.POINTER(_vp)]),
    "mphy_solver_destroy": (C.c_int, [_vp]),
    "mphy_solver_get_state": (C.c_int, [_vp, _i32]),
    "mphy_solver_zero": (C.c_int, [_vp]),
    "mphy_solver_assemble": (C.c_int, [_vp, _vp, _i64]),
    "mphy_solver_assemble_batch": (C.c_int, [_vp, C.c_int32, _vp, _vp, _vp]),
    "mphy_solver_assemble_batch_host": (C.c_int, [_vp, C.c_int32, _i32, _d, _d]),
    "mphy_solver_add_nodal_forces": (C.c_int, [_vp, _vp, C.c_double]),
    "mphy_solver_add_nodal_forces_host": (C.c_int, [_vp, _d, C.c_double]),
    "mphy_solver_rhs_norm": (C.c_int, [_vp, _d]),
    "mphy_solver_solve": (C.c_int, [_vp, _i32, _d]),
    "mphy_solver_spmv": (C.c_int, [_vp, _vp, _vp]),
    "mphy_solver_spmv_dot": (C.c_int, [_vp, _vp, _vp, _d]),
    "mphy_solver_matrix_info": (C.c_int, [_vp, _i64, _i64, _i64]),
    "mphy_solver_pc_pattern": (C.c_int, [_vp, _i64, _i64, _i32]),
    "mphy_solver_pc_get_blocks": (C.c_int, [_vp, _vp]),
    "mphy_solver_pc_set_blocks": (C.c_int, [_vp, _vp]),
    "mphy_solver_pc_setup": (C.c_int, [_vp, _i32]),
    "mphy_solver_true_residual": (C.c_int, [_vp, _d]),
    "mphy_gnn_param_count": (C.c_int, []),
    "mphy_gnn_create": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(_vp)]),
    "mphy_gnn_destroy": (C.c_int, [_vp]),
    "mphy_gnn_get_params": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "mphy_gnn_set_params": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "mphy_gnn_loss_and_grads": (C.c_int, [_vp, _vp, _d, C.POINTER(C.c_float)]),
    "mphy_gnn_train_step": (C.c_int, [_vp, _vp, C.c_float, _d]),
    "mphy_gnn_predict": (C.c_int, [_vp, _vp, C.POINTER(C.c_float)]),
    "mphy_solver_attach_gnn": (C.c_int, [_vp, _vp]),
    "mphy_solver_pc_last": (C.c_int, [_vp, _i32, C.POINTER(C.c_float), _i32, _i32, _d]),
    "mphy_solver_coarse_info": (C.c_int, [_vp, _i32, _i32, C.POINTER(C.c_float)]),
    "mphy_solver_get_solution": (C.c_int, [_vp, _vp]),
    "mphy_solver_get_solution_host": (C.c_int, [_vp, _d]),
    "mphy_solver_update_disp": (C.c_int, [_vp, _vp]),
    "mphy_solver_export": (C.c_int, [_vp, _d, _d, _d]),
    "mphy_solver_set_mixed_p0": (C.c_int, [_vp, C.c_int32]),
    "mphy_solver_p0_pressure": (C.c_int, [_vp, _d, _d]),
    "mphy_solver_save_step": (C.c_int, [_vp, _vp]),
    "mphy_newton_iteration": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_double, C.POINTER(IterStats)]),
    "mphy_newton_iteration_host": (C.c_int, [_vp, _d, _d, C.c_double, C.c_double, C.POINTER(IterStats)]),
    "mphy_newton_run": (C.c_int, [_vp, _d, C.POINTER(NewtonOpts), _d, C.POINTER(IterStats), C.c_int32, _i32]),
    "mphy_arclength_run": (C.c_int, [_vp, _d, C.POINTER(NewtonOpts), _d, _d, C.c_int32, _i32, C.POINTER(IterStats),
                                     _d, C.c_int32, _i32]),
    "mphy_mixed_opts_default": (None, [C.POINTER(MixedOpts)]),
    "mphy_mixed_create": (C.c_int, [_vp, _vp, _vp, C.POINTER(MixedOpts), C.POINTER(_vp)]),
    "mphy_mixed_destroy": (C.c_int, [_vp]),
    "mphy_mixed_info": (C.c_int, [_vp, _i32, _i64, _i64]),
    "mphy_mixed_pressure_nodes": (C.c_int, [_vp, _i32]),
    "mphy_mixed_elem_eval": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64]),
    "mphy_mixed_assemble": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, _vp, _d, _i64]),
    "mphy_mixed_apply": (C.c_int, [_vp, _vp, _vp]),
    "mphy_mixed_vectors": (C.c_int, [_vp, _vp, _vp, _vp]),
    "mphy_mixed_solve": (C.c_int, [_vp, _i32, _d]),
    "mphy_mixed_newton_run": (C.c_int, [_vp, _d, C.POINTER(NewtonOpts), _d, _d, C.POINTER(IterStats), C.c_int32,
                                        _i32]),
    "mphy_batch_create": (C.c_int, [_vp, C.c_int32, _i32, C.POINTER(_vp)]),
    "mphy_batch_destroy": (C.c_int, [_vp]),
    "mphy_batch_set_schedule": (C.c_int, [_vp, C.c_int32, C.c_int32]),
    "mphy_batch_get_schedule": (C.c_int, [_vp, _i32, _i32]),
    "mphy_batch_set_coarse": (C.c_int, [_vp, C.c_int32]),
    "mphy_batch_autotune": (C.c_int, [_vp, C.c_int32, C.c_int32, _i32, _i32, _i32, C.POINTER(C.c_float)]),
    "mphy_batch_solve": (C.c_int, [_vp, C.c_int32, _i32, _i32, _d, C.POINTER(C.c_float)]),
    "mphy_batch_instance_info": (C.c_int, [_vp, _i32, _i32, _i32, _d]),
    "mphy_batch_newton_run": (C.c_int, [_vp, _d, C.POINTER(NewtonOpts), _d, _i32, _i32, _i32, C.POINTER(BatchStats)]),
}

_lib = None


def load(path: str | None = None):
    """Load libmphy.so once. Raises OSError when it is missing (no fallback exists)."""
    global _lib
    if _lib is None:
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise OSError(f"{p} is not built; run `python -m mphyfem_b200.build`")
        L = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_string(status: int) -> str:
    try:
        return load().mphy_status_string(status).decode()
    except OSError:
        return "?"


def check(rc: int, allow=()) -> int:
    if rc != OK and rc not in allow:
        raise MphyError(rc, load().mphy_last_error().decode())
    return rc
