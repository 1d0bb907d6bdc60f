"""Loader of the in-tree CUDA library (``libifea_gpu.so``) and its C-ABI signatures (include/ifea_gpu.h).

There is no CPU fallback: if the library is missing or no CUDA device is usable, calls raise.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libifea_gpu.so")

STATUS = {0: "IFEA_OK", 1: "IFEA_INPUT_INVALID", 2: "IFEA_DIVERGED", 3: "IFEA_MESH_DISTORTED", 4: "IFEA_NOT_SPD",
          5: "IFEA_BAD_STATE", 6: "IFEA_CUDA_ERROR", 7: "IFEA_CANCELLED"}


class IfeaError(RuntimeError):
    """A failed C-ABI call; ``status`` maps to the reference's exception type."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class InputValidationError(IfeaError): pass          # InputValidationException
class SolverDivergenceError(IfeaError): pass         # SolverDivergenceException
class MeshDistortionError(IfeaError): pass           # MeshDistortionException
class MatrixNotPositiveDefiniteError(IfeaError): pass  # MatrixNotPositiveDefiniteException
class EngineUnavailableError(IfeaError): pass        # EngineUnavailableException


_ERRORS = {1: InputValidationError, 2: SolverDivergenceError, 3: MeshDistortionError,
           4: MatrixNotPositiveDefiniteError, 6: EngineUnavailableError}


def raise_for(status, message):
    if status != 0:
        raise _ERRORS.get(status, IfeaError)(status, message)


class Params3D(C.Structure):
    _fields_ = [("C", C.c_double), ("N", C.c_double), ("M", C.c_double), ("eps0", C.c_double),
                ("friction", C.c_double), ("ram", C.c_double), ("h", C.c_double), ("ds", C.c_double),
                ("tol", C.c_double), ("max_iter", C.c_int32), ("auto_step", C.c_int32), ("max_cutbacks", C.c_int32),
                ("remesh_quality", C.c_double), ("size", C.c_double), ("sym_x", C.c_int32), ("sym_y", C.c_int32),
                ("sym_factor", C.c_int32), ("penalty_factor", C.c_double), ("newton_blend", C.c_double),
                ("quadratic_ls", C.c_int32), ("extrapolate_start", C.c_int32), ("adaptive_newton", C.c_int32),
                ("sticky_secant", C.c_int32), ("pcg_budget", C.c_int32)]


class Params2D(C.Structure):
    _fields_ = [("C", C.c_double), ("N", C.c_double), ("M", C.c_double), ("eps0", C.c_double),
                ("friction", C.c_double), ("ram", C.c_double), ("ds", C.c_double), ("tol", C.c_double),
                ("max_iter", C.c_int32), ("axisymmetric", C.c_int32), ("length", C.c_double), ("radius", C.c_double),
                ("height", C.c_double), ("nx", C.c_int32), ("nz", C.c_int32)]


class StepInfo(C.Structure):
    _fields_ = [("step", C.c_int32), ("iterations", C.c_int32), ("load", C.c_double), ("reaction", C.c_double),
                ("stroke", C.c_double), ("gap", C.c_double), ("time", C.c_double), ("dt", C.c_double),
                ("volume_change_pct", C.c_double), ("last_rel", C.c_double), ("n_factor", C.c_int32),
                ("n_pcg", C.c_int32), ("remesh_requests", C.c_int32), ("cutbacks", C.c_int32)]


_vp, _dp, _i32p, _u8p, _i64p = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_uint8), C.POINTER(C.c_int64)
_st = C.c_int
_fp = C.POINTER(C.c_float)
class DieGrid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("x0", C.c_double), ("y0", C.c_double), ("dx", C.c_double),
                ("h", C.POINTER(C.c_double))]


class RemeshArgs(C.Structure):
    _fields_ = [("nn", C.c_int32), ("ne", C.c_int32), ("x", C.POINTER(C.c_double)), ("tets", C.POINTER(C.c_int32)),
                ("vg", C.POINTER(C.c_double)), ("eps", C.POINTER(C.c_double)), ("dmg", C.POINTER(C.c_double)),
                ("sig", C.POINTER(C.c_double)), ("rate", C.POINTER(C.c_double)), ("mean", C.POINTER(C.c_double)),
                ("bottom", DieGrid), ("top", DieGrid), ("gap", C.c_double), ("h", C.c_double), ("vol_target", C.c_double),
                ("sym_x", C.c_int32), ("sym_y", C.c_int32), ("recovery_pass", C.c_int32),
                ("refinement_levels", C.c_int32), ("max_nodes", C.c_int32), ("sig_ref", C.c_double),
                ("n_hot", C.c_int32), ("hot", C.POINTER(C.c_double))]


INSIDE_FN = C.CFUNCTYPE(C.c_int32, C.c_double, C.c_double, C.c_double, C.c_void_p)
SIZE_FN = C.CFUNCTYPE(C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p)

SIGNATURES = {
    "ifea3d_create": (_st, [C.POINTER(Params3D), C.POINTER(_vp)]),
    "ifea3d_destroy": (None, [_vp]),
    "ifea3d_last_error": (C.c_char_p, [_vp]),
    "ifea3d_set_mesh": (_st, [_vp, C.c_int32, C.c_int32, _dp, _i32p, _u8p, _u8p]),
    "ifea3d_set_die": (_st, [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, _dp]),
    "ifea3d_set_trimesh_die": (_st, [_vp, C.c_int32, C.c_int32, _dp, C.c_int32, _i32p]),
    "ifea3d_die_query": (_st, [_vp, C.c_int32, C.c_int32, _dp, C.c_double, _dp, _dp, _dp, _dp]),
    "ifea3d_init": (_st, [_vp] + [C.c_double] * 6),
    "ifea3d_step": (_st, [_vp, C.POINTER(StepInfo), _i32p]),
    "ifea3d_pattern_size": (_st, [_vp, _i64p, _i32p]),
    "ifea3d_get_pattern": (_st, [_vp, _i32p, _i32p]),
    "ifea3d_prepare_step": (_st, [_vp]),
    "ifea3d_assemble": (_st, [_vp, C.c_int32, C.c_int32, _dp, _dp, _dp]),
    "ifea3d_apply_bc": (_st, [_vp, _dp]),
    "ifea3d_solve_velocity": (_st, [_vp, _i32p, _i32p, _i32p]),
    "ifea3d_final_evaluation": (_st, [_vp, _dp, _dp]),
    "ifea3d_try_update": (_st, [_vp, C.c_double, _i32p]),
    "ifea3d_set_warm": (_st, [_vp, C.c_int32]),
    "ifea3d_set_stream": (_st, [_vp, _vp]),
    "ifea3d_get_array": (_st, [_vp, C.c_char_p, _vp, C.c_int64]),
    "ifea3d_array_size": (_st, [_vp, C.c_char_p, _i64p, _i32p]),
    "ifea3d_set_array": (_st, [_vp, C.c_char_p, _vp, C.c_int64]),
    "ifea3d_get_scalar": (_st, [_vp, C.c_char_p, _dp]),
    "ifea3d_set_scalar": (_st, [_vp, C.c_char_p, C.c_double]),
    "ifea_spd_create": (_st, [C.POINTER(_vp)]),
    "ifea_spd_destroy": (None, [_vp]),
    "ifea_spd_last_error": (C.c_char_p, [_vp]),
    "ifea_spd_analyze": (_st, [_vp, C.c_int32, _i32p, _i32p]),
    "ifea_spd_factorize": (_st, [_vp, _dp]),
    "ifea_spd_solve": (_st, [_vp, _dp, _dp]),
    "ifea_spd_factor_nonzeros": (C.c_int64, [_vp]),
    "ifea_spd_name": (C.c_char_p, [_vp]),
    "ifea2d_create": (_st, [C.POINTER(Params2D), C.c_int32, _dp, C.c_int32, _dp, C.POINTER(_vp)]),
    "ifea2d_destroy": (None, [_vp]),
    "ifea2d_last_error": (C.c_char_p, [_vp]),
    "ifea2d_step": (_st, [_vp, C.POINTER(StepInfo), _i32p]),
    "ifea2d_prepare": (_st, [_vp]),
    "ifea2d_assemble": (_st, [_vp, C.c_int32, C.c_int32, _dp, _dp, _dp]),
    "ifea2d_solve_velocity": (_st, [_vp, C.c_int32, _i32p, _i32p]),
    "ifea2d_get_array": (_st, [_vp, C.c_char_p, _vp, C.c_int64]),
    "ifea2d_array_size": (_st, [_vp, C.c_char_p, _i64p, _i32p]),
    "ifea2d_get_scalar": (_st, [_vp, C.c_char_p, _dp]),
    "ifea_band_factor_solve": (_st, [C.c_int32, C.c_int32, _dp, _dp, _i32p, _dp]),
    "ifea_band_factor_solve_noalloc": (_st, [C.c_int32, C.c_int32, _vp, _vp, _i32p, _dp, _vp]),
    "ifea_version": (C.c_char_p, []),
    "ifea_mlp_create": (_st, [C.c_uint64, C.POINTER(_vp)]),
    "ifea_mlp_destroy": (None, [_vp]),
    "ifea_mlp_last_error": (C.c_char_p, [_vp]),
    "ifea_mlp_param_count": (C.c_int64, []),
    "ifea_mlp_get_params": (_st, [_vp, _fp, C.c_int64]),
    "ifea_mlp_set_params": (_st, [_vp, _fp, C.c_int64]),
    "ifea_mlp_get_normalisation": (_st, [_vp, _fp]),
    "ifea_mlp_set_normalisation": (_st, [_vp, _fp]),
    "ifea_mlp_add_samples": (_st, [_vp, _fp, _fp, C.c_int64]),
    "ifea_mlp_samples": (C.c_int64, [_vp]),
    "ifea_mlp_clear_samples": (_st, [_vp]),
    "ifea_mlp_fit_normalisation": (_st, [_vp]),
    "ifea_mlp_forward": (_st, [_vp, _fp, C.c_int64, _fp]),
    "ifea_mlp_gradients": (_st, [_vp, _fp, _fp, C.c_int64, _fp, _fp]),
    "ifea_mlp_train": (_st, [_vp, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _fp, _dp]),
    "ifea3d_set_warm_start": (_st, [_vp, _vp, C.c_int32]),
    "ifea3d_last_remesh": (C.c_char_p, [_vp]),
    "ifea3d_set_cavity": (_st, [_vp, C.c_int32, _dp]),
    "ifea3d_fill_percent": (_st, [_vp, _dp]),
    "ifea_batch_create": (_st, [C.c_int32, C.POINTER(_vp), C.c_int32, C.POINTER(_vp), C.c_int32, C.POINTER(_vp)]),
    "ifea_batch_step": (_st, [_vp, C.c_int32, C.POINTER(StepInfo), _i32p]),
    "ifea_batch_destroy": (None, [_vp]),
    "ifea3d_autotune": (_st, [_vp, C.c_int32, _dp, _dp, _dp]),
    "ifea3d_time_factor_solve": (_st, [_vp, _dp]),
    "ifea_tetmesh_stuff": (_st, [INSIDE_FN, _vp, _dp, _dp, C.c_double, C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "ifea_tetmesh_refine": (_st, [_vp, SIZE_FN, _vp, C.c_int32, _i32p]),
    "ifea_tetmesh_node_count": (C.c_int32, [_vp]),
    "ifea_tetmesh_tet_count": (C.c_int32, [_vp]),
    "ifea_tetmesh_get": (_st, [_vp, _dp, _i32p]),
    "ifea_tetmesh_destroy": (None, [_vp]),
    "ifea_remesh_workpiece": (_st, [C.POINTER(RemeshArgs), C.POINTER(_vp)]),
    "ifea_remesh_node_count": (C.c_int32, [_vp]),
    "ifea_remesh_tet_count": (C.c_int32, [_vp]),
    "ifea_remesh_why": (C.c_char_p, [_vp]),
    "ifea_remesh_get": (_st, [_vp, _dp, _i32p, _u8p, _u8p, _u8p, _dp, _dp, _dp, _dp, _dp, _dp]),
    "ifea_remesh_destroy": (None, [_vp]),
}

_LIB = None


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise EngineUnavailableError(6, f"{LIB_PATH} is missing; run impressionfea_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            if not hasattr(L, name):
                continue
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB
