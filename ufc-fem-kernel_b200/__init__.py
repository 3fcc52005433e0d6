"""B200 (sm_100a) implementation of UFC's implicit-static C3D8 hot path.

The compute path is libufc_gpu.so (hand-written CUDA, C-ABI in
include/ufc_gpu.h); this package is its Python host side:

* :mod:`.fem`      -- `FemModel`, one GPU context per model (mesh, pattern,
  assembly, internal force, Jacobi-PCG, Newton increments, adjoint kernel);
* :mod:`.ufc_api`  -- the reference's call surface (Desc/State/Algo/Ctx
  bundles and routine names of ufc_core L2/L4/L5) over `FemModel`;
* :mod:`.adjoint`  -- `UfcLinearElastic`, a torch.autograd.Function with the
  hand-written adjoint;
* :mod:`.mesh`     -- seeded structured meshes, Dirichlet sets and loads.
"""
from . import _abi, mesh, ufc_api  # noqa: F401
from ._abi import LibraryMissing, check_abi, load  # noqa: F401
from .fem import FemModel, NrResult, SolverAlgo, SolverState, StepResult, UfcError, lifted_rhs  # noqa: F401

PRECISION_FP64 = _abi.PRECISION_FP64
PRECISION_FP32_REFINE = _abi.PRECISION_FP32_REFINE
PRECISION_FP32_MATRIX = _abi.PRECISION_FP32_MATRIX
ACCUMULATE_STORAGE = _abi.ACCUMULATE_STORAGE
ACCUMULATE_FP64 = _abi.ACCUMULATE_FP64
BUILD_FP64 = _abi.BUILD_FP64
BUILD_FP32 = _abi.BUILD_FP32
BUILD_FP32_ROUNDED = _abi.BUILD_FP32_ROUNDED
BUILD_FP32_DIFF = _abi.BUILD_FP32_DIFF
BUILD_SYMMETRIC = _abi.BUILD_SYMMETRIC
REFINE_KEEP_DIRECTION = _abi.REFINE_KEEP_DIRECTION
REFINE_RESTART = _abi.REFINE_RESTART
REFINE_FORCE_FP32 = _abi.REFINE_FORCE_FP32
MAT_ELASTIC_ISO = _abi.MAT_ELASTIC_ISO
MAT_J2_ISO = _abi.MAT_J2_ISO
SOLV_PREC_JACOBI = _abi.SOLV_PREC_JACOBI
SOLV_PREC_MG = _abi.SOLV_PREC_MG
STATUS_OK = _abi.STATUS_OK
STATUS_INVALID = _abi.STATUS_INVALID
STATUS_NOT_CONVERGED = _abi.STATUS_NOT_CONVERGED
