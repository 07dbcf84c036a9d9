"""ctypes binding of libgrico_b200.so (declarations mirror include/grico_b200.h).

The library is the only compute path: if it is missing, or no CUDA device is present when a
plan is created, calls raise instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgrico_b200.so")

GRICO_OK = 0
GRICO_ERR_INVALID = -1
GRICO_ERR_UNSUPPORTED_FORM = -2
GRICO_ERR_NOT_CONVERGED = -3
GRICO_ERR_NONFINITE = -4
GRICO_ERR_BREAKDOWN = -5
GRICO_ERR_CUDA = -6
GRICO_ERR_NO_DEVICE = -7
GRICO_ERR_TIMEOUT = -8

GRICO_BASIS_FULL = 0
GRICO_BASIS_TRUNK = 1
GRICO_CONTINUITY_CG = 0
GRICO_CONTINUITY_DG = 1
GRICO_FORM_MASS_DIFFUSION = 1
GRICO_ITEM_CELL = 1
GRICO_ITEM_NITSCHE = 2
GRICO_ITEM_SUBCELLS = 3
GRICO_ITEM_INTERFACE = 4
# (modes per axis, points per axis) pairs the subcell kernel is compiled for, per dimension
SUBCELL_SHAPES = {3: {(2, 2), (2, 3), (3, 3), (2, 4), (3, 4), (4, 4)},
                  2: {(n, q) for n in range(2, 9) for q in (n, n + 1) if q <= 8}}
GRICO_PREC_FP64 = 0
GRICO_PREC_FP32 = 1
# 3-D tensor-kernel variants accepted by grico_plan_set_tiles (0..TILE_VARIANTS-1)
TILE_VARIANTS = 11
GRICO_FLAG_HOST_POINTERS = 1
GRICO_FLAG_NO_GRAPH = 2
GRICO_FLAG_MIXED = 4
GRICO_FLAG_TIME_BATCHES = 8
GRICO_FLAG_ASYNC = 16
GRICO_FLAG_DETERMINISTIC = 32
GRICO_PRECOND_IDENTITY = 0
GRICO_PRECOND_JACOBI = 1
GRICO_PRECOND_MULTIGRID = 2
GRICO_SMOOTHER_JACOBI = 0
GRICO_SMOOTHER_CHEBYSHEV = 1
GRICO_SMOOTHER_GMRES = 2

P = C.c_void_p
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)


class GricoCellBatchDesc(C.Structure):
    _fields_ = [
        ("n_cells", C.c_int32),
        ("degree", C.c_int32 * 3),
        ("qpoints", C.c_int32 * 3),
        ("map_index", i32p),
        ("map_coef", f64p),
        ("n_tail", C.c_int64),
        ("tail_offsets", i64p),
        ("tail_index", i32p),
        ("tail_coef", f64p),
        ("cell_size", f64p),
        ("kappa_points", f64p),
    ]


class GricoPointBatchDesc(C.Structure):
    _fields_ = [
        ("n_items", C.c_int32),
        ("kind", C.c_int32),
        ("degree", C.c_int32 * 3),
        ("map_index", i32p),
        ("map_coef", f64p),
        ("n_tail", C.c_int64),
        ("tail_offsets", i64p),
        ("tail_index", i32p),
        ("tail_coef", f64p),
        ("cell_size", f64p),
        ("point_offsets", i64p),
        ("ref_points", f64p),
        ("weights", f64p),
        ("normals", f64p),
        ("eta", f64p),
        ("kappa_points", f64p),
        ("qpoints", C.c_int32 * 3),
        ("subcell_offsets", i64p),
        ("subcell_level", i32p),
        ("subcell_pos", i32p),
        ("subcell_mask", C.POINTER(C.c_uint64)),
        ("subcell_weight", f64p),
        ("degree_plus", C.c_int32 * 3),
        ("ref_points_plus", f64p),
        ("cell_size_plus", f64p),
        ("face_axis", i32p),
    ]


class GricoPlanDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("form", C.c_int32),
        ("mass", C.c_double),
        ("kappa", C.c_double),
        ("n_full", C.c_int64),
        ("n_batches", C.c_int32),
        ("batches", C.POINTER(GricoCellBatchDesc)),
        ("n_fixed", C.c_int64),
        ("fixed_dofs", i64p),
        ("fixed_values", f64p),
        ("n_relations", C.c_int64),
        ("rel_pivot", i64p),
        ("rel_offsets", i64p),
        ("rel_index", i64p),
        ("rel_coef", f64p),
        ("rel_rhs", f64p),
        ("n_reduced", C.c_int64),
        ("red_offsets", i64p),
        ("red_index", i64p),
        ("red_coef", f64p),
        ("red_shift", f64p),
        ("n_point_batches", C.c_int32),
        ("point_batches", C.POINTER(GricoPointBatchDesc)),
    ]


class GricoSolveOptions(C.Structure):
    _fields_ = [
        ("relative_tolerance", C.c_double),
        ("absolute_tolerance", C.c_double),
        ("maxiter", C.c_int32),
        ("preconditioner", C.c_int32),
        ("restart", C.c_int32),
        ("use_initial", C.c_int32),
    ]


class GricoSolveReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("status", C.c_int32),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("seconds", C.c_double),
    ]


class GricoTransferDesc(C.Structure):
    _fields_ = [
        ("n_fine", C.c_int64),
        ("n_coarse", C.c_int64),
        ("row_offsets", i64p),
        ("col_index", i64p),
        ("values", f64p),
    ]


class GricoMGOptions(C.Structure):
    _fields_ = [
        ("smoother", C.c_int32),
        ("pre_steps", C.c_int32),
        ("post_steps", C.c_int32),
        ("jacobi_omega", C.c_double),
        ("chebyshev_degree", C.c_int32),
        ("chebyshev_lower", C.c_double),
        ("precision", C.c_int32),
        ("smoother_restart", C.c_int32),
    ]


# name -> (restype, argtypes); every symbol include/grico_b200.h declares
class GricoLearnedDesc(C.Structure):
    _fields_ = [
        ("level", C.c_int32),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("grid_index", i64p),
        ("grid_log_coefficient", C.POINTER(C.c_float)),
        ("n_layers", C.c_int32),
        ("channels", i32p),
        ("weights", C.POINTER(C.POINTER(C.c_float))),
        ("biases", C.POINTER(C.POINTER(C.c_float))),
        ("omega", C.c_double),
    ]


SIGNATURES = {
    "grico_space_build": (C.c_int, [C.c_int, i64p, C.c_int64, i32p, i64p, i32p, C.c_int, C.c_int, C.c_int, C.POINTER(P)]),
    "grico_space_destroy": (C.c_int, [P]),
    "grico_space_sizes": (C.c_int, [P, i64p, i64p, i64p, i64p, i64p]),
    "grico_space_export": (C.c_int, [P, i64p, i64p, i64p, i64p, f64p, i32p, i64p, i32p, i32p, i64p, i64p, i32p]),
    "grico_transfer_build": (C.c_int, [P, P, i64p, i64p, f64p, C.c_int64, i64p, C.c_int64, C.POINTER(P)]),
    "grico_transfer_export": (C.c_int, [P, i64p, i64p, i64p, f64p]),
    "grico_transfer_destroy": (C.c_int, [P]),
    "grico_gauss_legendre": (C.c_int, [C.c_int, f64p, f64p]),
    "grico_fe_basis": (C.c_int, [C.c_double, C.c_int, f64p, f64p]),
    "grico_plan_create": (C.c_int, [C.POINTER(GricoPlanDesc), C.POINTER(P)]),
    "grico_plan_destroy": (C.c_int, [P]),
    "grico_plan_sizes": (C.c_int, [P, i64p, i64p]),
    "grico_apply": (C.c_int, [P, P, P, C.c_int, C.c_int, C.c_int, P]),
    "grico_reduced_apply": (C.c_int, [P, P, P, C.c_int, C.c_int, C.c_int, P]),
    "grico_reduced_rhs": (C.c_int, [P, C.POINTER(f64p), f64p, C.c_int]),
    "grico_rhs": (C.c_int, [P, C.POINTER(f64p), f64p, C.c_int]),
    "grico_reduced_rhs_static": (C.c_int, [P, C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p]),
    "grico_reduced_diagonal": (C.c_int, [P, f64p, C.c_int]),
    "grico_expand_reduced": (C.c_int, [P, f64p, f64p, C.c_int]),
    "grico_cg_solve": (C.c_int, [P, P, f64p, f64p, C.POINTER(GricoSolveOptions), C.POINTER(GricoSolveReport), C.c_int]),
    "grico_fgmres_solve": (C.c_int, [P, P, f64p, f64p, C.POINTER(GricoSolveOptions), C.POINTER(GricoSolveReport), C.c_int]),
    "grico_mg_create": (C.c_int, [C.POINTER(P), C.c_int, C.POINTER(GricoTransferDesc), f64p, C.POINTER(GricoMGOptions), C.POINTER(P)]),
    "grico_mg_destroy": (C.c_int, [P]),
    "grico_mg_vcycle": (C.c_int, [P, f64p, f64p, C.c_int]),
    "grico_mg_lambda_max": (C.c_double, [P, C.c_int]),
    "grico_mg_set_learned": (C.c_int, [P, C.POINTER(GricoLearnedDesc)]),
    "grico_plan_autotune": (C.c_int, [P, C.c_int, C.c_int, C.c_int, i32p]),
    "grico_plan_set_tiles": (C.c_int, [P, C.c_int, i32p, C.c_int]),
    "grico_plan_batch_times": (C.c_int, [P, f64p, i64p, C.c_int]),
    "grico_plan_set_mass_points": (C.c_int, [P, C.POINTER(f64p), C.c_int]),
    "grico_eval_points": (C.c_int, [P, f64p, C.c_int, C.POINTER(f64p), C.c_int]),
    "grico_cg_solve_multi": (C.c_int, [P, f64p, f64p, C.c_int, C.POINTER(GricoSolveOptions), C.POINTER(GricoSolveReport), C.c_int]),
    "grico_mg_learned_stats": (C.c_int, [P, i64p, i64p]),
    "grico_conv3d_forward": (C.c_int, [P, C.c_int, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, P]),
    "grico_conv_tc_weight_bytes": (C.c_int64, [C.c_int, C.c_int]),
    "grico_conv3d_pack_weights_tc": (C.c_int, [P, C.c_int, C.c_int, P, P]),
    "grico_conv3d_forward_tc": (C.c_int, [P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, P]),
    "grico_conv_tc_status": (C.c_int, [P]),
    "grico_tc_status": (C.c_int, [P]),
    "grico_conv3d_backward_data": (C.c_int, [P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P]),
    "grico_conv3d_backward_weight": (C.c_int, [P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P]),
    "grico_relu_backward": (C.c_int, [P, P, C.c_int64, P]),
    "grico_mse_grad": (C.c_int, [P, P, P, P, C.c_int64, C.c_double, P, P, P]),
    "grico_adam_step": (C.c_int, [P, P, P, P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_int, C.c_float, P]),
    "grico_grid_gather": (C.c_int, [P, C.c_int64, P, C.c_float, P, P]),
    "grico_grid_scatter_add": (C.c_int, [P, C.c_int64, P, C.c_float, P, P]),
    "grico_weighted_residual": (C.c_int, [P, P, P, P, C.c_int64, P, P, P]),
    "grico_halo_pack": (C.c_int, [P, P, P, C.c_int64, P, C.c_int64, P]),
    "grico_halo_unpack": (C.c_int, [P, P, P, C.c_int64, P, P]),
    "grico_vec_dot": (C.c_int, [C.c_int64, P, P, P, P, P]),
    "grico_vec_axpby": (C.c_int, [C.c_int64, C.c_double, P, C.c_double, P, P]),
    "grico_vec_invert": (C.c_int, [C.c_int64, P, P, P]),
    "grico_cg_update_xr": (C.c_int, [C.c_int64, C.c_int64, P, P, P, P, P, P, P]),
    "grico_cg_precondition": (C.c_int, [C.c_int64, C.c_int64, P, P, P, P, P, P]),
    "grico_cg_direction": (C.c_int, [C.c_int64, P, P, P, P]),
    "grico_last_error": (C.c_char_p, []),
}

_lib = None


def lib():
    """Load the in-tree shared library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libgrico_b200.so is not built ({LIB_PATH}); run grico.jl_b200/build.py")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class GricoError(ValueError):
    """Raised for every non-zero status; the reference raises ArgumentError in these cases."""

    def __init__(self, code, message):
        super().__init__(f"{message} (status {code})")
        self.code = code


def check(code, what=""):
    if code != GRICO_OK:
        msg = lib().grico_last_error()
        msg = msg.decode() if msg else ""
        raise GricoError(code, f"{what}: {msg}" if what else msg)
    return code


def ptr(array, ctype):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if array is None:
        return None
    return array.ctypes.data_as(C.POINTER(ctype))
