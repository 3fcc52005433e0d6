"""ctypes mirror of include/ufc_gpu.h (the C-ABI of libufc_gpu.so).

The struct layouts below follow the header field by field; `check_abi()`
verifies that every function the header declares is exported.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libufc_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "ufc_gpu.h")

# IF_STATUS_* (ufc_core/L1_IF/Error/IF_Err_Brg.f90:95-110)
STATUS_OK = 0
STATUS_INVALID = 1
STATUS_ERROR = 2
STATUS_CONVERGED = 3
STATUS_NOT_CONVERGED = 4
STATUS_NOT_FOUND = 5
STATUS_WARN = 6
STATUS_MEM_ERROR = 7
STATUS_IO_ERROR = 8
STATUS_EXISTS = 9
STATUS_FATAL = 10
STATUS_UNSUPPORTED = 11
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "ERROR", 3: "CONVERGED", 4: "NOT_CONVERGED", 5: "NOT_FOUND", 6: "WARN",
                7: "MEM_ERROR", 8: "IO_ERROR", 9: "EXISTS", 10: "FATAL", 11: "UNSUPPORTED"}

MEM_HOST = 0
MEM_DEVICE = 1
MAT_ELASTIC_ISO = 101
MAT_J2_ISO = 201
SOLV_METHOD_CG = 3
SOLV_PREC_NONE = 0
SOLV_PREC_JACOBI = 1
SOLV_PREC_MG = 5
PRECISION_FP64 = 0
PRECISION_FP32_REFINE = 1
PRECISION_FP32_MATRIX = 2
ACCUMULATE_STORAGE = 0
ACCUMULATE_FP64 = 1
BUILD_FP64 = 1
BUILD_FP32 = 2
BUILD_FP32_ROUNDED = 4
BUILD_FP32_DIFF = 8
BUILD_SYMMETRIC = 16
REFINE_KEEP_DIRECTION = 0
REFINE_RESTART = 1
REFINE_FORCE_FP32 = 2

_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_d = C.c_double


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", _i32), ("n_elems", _i32), ("coords", _p), ("conn", _p), ("index_base", _i32),
                ("mem", _i32)]


class MaterialDesc(C.Structure):
    _fields_ = [("mat_model_id", _i32), ("nprops", _i32), ("per_element", _i32), ("props", _p), ("mem", _i32)]


class BcDesc(C.Structure):
    _fields_ = [("n_fixed", _i32), ("dofs", _p), ("values", _p), ("mem", _i32)]


class PatternInfo(C.Structure):
    _fields_ = [("n_dof", _i64), ("nnz", _i64), ("nnzb", _i64), ("sell_blocks", _i64), ("n_colors", _i32),
                ("max_row_blocks", _i32)]


class CsrExportArg(C.Structure):
    _fields_ = [("index_base", _i32), ("mem", _i32), ("row_ptr", _p), ("col_ind", _p), ("values", _p),
                ("values32", _p)]


class ElemKeArg(C.Structure):
    _fields_ = [("build", _i32), ("status", _i32), ("elapsed_ms", _d)]


class ElemFeArg(C.Structure):
    _fields_ = [("u", _p), ("f_ext", _p), ("fint", _p), ("r", _p), ("mem", _i32), ("update_state", _i32),
                ("rnorm", _d), ("fint_norm", _d), ("status", _i32)]


class MatUpdateArg(C.Structure):
    _fields_ = [("mat_model_id", _i32), ("n_points", _i32), ("nprops", _i32), ("props_per_point", _i32),
                ("props", _p), ("stress_n", _p), ("dstrain", _p), ("sdv_n", _p), ("stress", _p), ("sdv", _p),
                ("ddsdde", _p), ("yielded", _p), ("mem", _i32), ("status", _i32)]


class SolverAlgo(C.Structure):
    _fields_ = [("method", _i32), ("precond_type", _i32), ("max_iter", _i32), ("precision_mode", _i32),
                ("tolerance", _d), ("abs_tolerance", _d), ("refine_delta", _d), ("check_every", _i32),
                ("use_x0", _i32), ("refine_policy", _i32), ("accumulate", _i32)]


class SolverState(C.Structure):
    _fields_ = [("niter", _i32), ("n_refine", _i32), ("converged", _i32), ("convergence_flag", _i32),
                ("rnorm", _d), ("initial_residual", _d), ("solve_time", _d), ("fp64_iters", _i32),
                ("reserved", _i32)]


class NrArg(C.Structure):
    _fields_ = [("u_prescribed", _p), ("f_ext", _p), ("mem", _i32), ("max_iterations", _i32),
                ("tolerance_force", _d), ("lin", SolverAlgo), ("iterations", _i32), ("converged", _i32),
                ("lin_iters_total", _i32), ("residual_norm", _d), ("res_hist", _d * 32), ("status", _i32)]


class StepArg(C.Structure):
    _fields_ = [("u_prescribed_end", _p), ("f_ext_start", _p), ("f_ext_end", _p), ("mem", _i32),
                ("time_period", _d), ("dt_initial", _d), ("dt_min", _d), ("dt_max", _d),
                ("max_increments", _i32), ("max_cutbacks", _i32), ("auto_dt", _i32), ("target_iters", _i32),
                ("growth_threshold", _d), ("growth_factor", _d), ("cutback_factor", _d),
                ("max_iterations", _i32), ("tolerance_force", _d), ("lin", SolverAlgo),
                ("hist_time", _p), ("hist_dt", _p), ("hist_iters", _p), ("hist_converged", _p),
                ("hist_cap", _i32), ("attempts", _i32), ("increments", _i32), ("cutbacks", _i32),
                ("nr_iterations", _i32), ("lin_iters_total", _i64), ("final_time", _d), ("completed", _i32),
                ("status", _i32)]


class MgArg(C.Structure):
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("max_levels", _i32), ("degree", _i32), ("ratio", _d),
                ("coarse_max", _i64), ("levels", _i32), ("precision", _i32), ("coarse_dof", _i64),
                ("setup_ms", _d)]


class FaceLoadArg(C.Structure):
    _fields_ = [("n_faces", _i32), ("elem", _p), ("face", _p), ("traction", _p), ("pressure", _p),
                ("index_base", _i32), ("mem", _i32), ("f", _p)]


class TimingInfo(C.Structure):
    _fields_ = [("spmv_launches", _i32), ("spmv_ms", _d), ("spmv_bytes", _i64), ("precision", _i32),
                ("kernel_launches", _i64)]


_SIGS = {
    "ufc_ctx_create": [_i32, C.POINTER(_p)],
    "ufc_ctx_destroy": [_p],
    "ufc_ctx_set_stream": [_p, _p],
    "ufc_ctx_set_instrument": [_p, _i32],
    "ufc_last_error": [_p, C.c_char_p, _i32],
    "ufc_mesh_set": [_p, C.POINTER(MeshDesc)],
    "ufc_material_set": [_p, C.POINTER(MaterialDesc)],
    "ufc_bc_set": [_p, C.POINTER(BcDesc)],
    "ufc_pattern_build": [_p, C.POINTER(PatternInfo)],
    "ufc_csr_export": [_p, C.POINTER(CsrExportArg)],
    "ufc_pattern_colors": [_p, _p, _i32, _i32],
    "ufc_elem_compute_ke": [_p, C.POINTER(ElemKeArg)],
    "ufc_elem_compute_fint": [_p, C.POINTER(ElemFeArg)],
    "ufc_mat_update_batch": [_p, C.POINTER(MatUpdateArg)],
    "ufc_stress_eval": [_p, _p, _p, _p, _i32],
    "ufc_spmv": [_p, _i32, _p, _p, _i32],
    "ufc_pcg_solve": [_p, _p, _p, _i32, C.POINTER(SolverAlgo), C.POINTER(SolverState)],
    "ufc_pcg_solve_block": [_p, _i32, _p, _p, _i32, C.POINTER(SolverAlgo), C.POINTER(SolverState)],
    "ufc_last_timing": [_p, C.POINTER(TimingInfo)],
    "ufc_last_residual_history": [_p, _p, _i32, C.POINTER(_i32)],
    "ufc_nr_increment": [_p, C.POINTER(NrArg)],
    "ufc_nr_step": [_p, C.POINTER(StepArg)],
    "ufc_mg_setup": [_p, C.POINTER(MgArg)],
    "ufc_mg_apply": [_p, _p, _p, _i32],
    "ufc_mg_level_info": [_p, _i32, C.POINTER(_i64), C.POINTER(_i64)],
    "ufc_mg_export": [_p, _i32, C.POINTER(CsrExportArg)],
    "ufc_load_faces": [_p, C.POINTER(FaceLoadArg)],
    "ufc_stress_nodal": [_p, _p, _p, _p, _i32],
    "ufc_reactions": [_p, _p, _p, _p, _i32],
    "ufc_state_commit": [_p],
    "ufc_state_rollback": [_p],
    "ufc_get_displacement": [_p, _p, _i32],
    "ufc_set_displacement": [_p, _p, _i32],
    "ufc_get_state": [_p, _p, _p, _p, _i32],
    "ufc_adjoint_sensitivity": [_p, _i32, _p, _p, _p, _i32],
    "ufc_csr_spmv_dot_noalloc": [_i64, _p, _p, _p, _p, _p, _p, _p, C.c_char_p, _i32],
}

_LIB = None


class LibraryMissing(RuntimeError):
    pass


def load(path: str | None = None):
    """Load libufc_gpu.so (built by the package's csrc/Makefile).  Raises
    LibraryMissing when it has not been built: there is no fallback path."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise LibraryMissing(f"{p} not found: build it with `make -C {os.path.join(HERE, 'csrc')}`")
    lib = C.CDLL(p)
    for name, args in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    if path is None:
        _LIB = lib
    return lib


def header_functions(header: str = HEADER):
    """Names of the functions include/ufc_gpu.h declares."""
    text = open(header).read()
    return sorted(set(re.findall(r"^int\s+(ufc_\w+)\s*\(", text, flags=re.M)))


def check_abi(lib=None):
    lib = lib or load()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    extra = [n for n in _SIGS if n not in header_functions()]
    return missing, extra
