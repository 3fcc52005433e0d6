"""The reference's call surface over FemModel: Desc/State/Algo/Ctx bundles and
routine names of ufc_core L2 (solver), L4 (element, material) and L5
(assembly, Newton-Raphson, step driver) for this path.

Each routine takes the bundles the reference routine takes, fills the INTENT
(OUT/INOUT) fields, and returns an ErrorStatusType instead of raising, as the
Fortran routines do (IF_STATUS_* codes of ufc_core/L1_IF/Error/IF_Err_Brg.f90:
95-110).  The work arrays of the reference's *_Ctx bundles live on the GPU
inside the FemModel, so every Ctx here carries the model (the ufc_ctx handle)
instead of r/p/Ap/z pointers.  One call replaces the whole loop the reference
routine runs: NM_Solver_PCG is one ufc_pcg_solve, RT_Asm_GlobalStiffness one
batched element loop and scatter, RT_NLSolver_NewtonRaph one device-resident
increment.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .fem import FemModel, SolverAlgo, UfcError

IF_STATUS_OK = A.STATUS_OK
IF_STATUS_INVALID = A.STATUS_INVALID
IF_STATUS_ERROR = A.STATUS_ERROR
IF_STATUS_NOT_CONVERGED = A.STATUS_NOT_CONVERGED
NM_SOLV_METHOD_CG = A.SOLV_METHOD_CG
NM_SOLV_PREC_NONE = A.SOLV_PREC_NONE
NM_SOLV_PREC_JACOBI = A.SOLV_PREC_JACOBI
NM_PREC_AMG = A.SOLV_PREC_MG


@dataclass
class ErrorStatusType:
    """ErrorStatusType (ufc_core/L1_IF/Error/IF_Err_Def.f90:118-135): the code
    and message every routine returns."""
    status_code: int = IF_STATUS_OK
    message: str = ""
    source: str = ""

    @property
    def ok(self):
        return self.status_code == IF_STATUS_OK


def init_error_status(status: ErrorStatusType | None = None) -> ErrorStatusType:
    status = status or ErrorStatusType()
    status.status_code, status.message, status.source = IF_STATUS_OK, "", ""
    return status


def _run(source, fn, *args, **kw):
    """(result, ErrorStatusType): the library's UfcError becomes a status."""
    try:
        return fn(*args, **kw), ErrorStatusType(IF_STATUS_OK, "", source)
    except UfcError as e:
        return None, ErrorStatusType(e.status_code, e.message, source)


# ---------------------------------------------------------------- L2 solver
@dataclass
class NM_Solver_Desc:
    """NM_Solver_Desc (ufc_core/L2_NM/Solver/NM_Solv_Def.f90:76-81)."""
    n: int = 0
    bandwidth: int = 0
    is_symmetric: bool = True
    is_spd: bool = True


class NM_Solver_Algo(SolverAlgo):
    """NM_Solver_Algo (NM_Solv_Def.f90:86-100): method, precond_type,
    max_iter, tolerance (relative to ||b||), plus this path's precision_mode
    (FP64, or FP32 iterations with FP64 residual refinement)."""

    def SetTolerance(self, tol):
        # NM_Solver_Algo_SetTol (NM_Solv_Def.f90:187-196) stops on tol <= 0
        if not tol > 0.0:
            raise ValueError("NM_Solver_Algo_SetTol: Tolerance must be positive")
        self.tolerance = float(tol)

    def SetMaxIter(self, max_iter):
        # NM_Solver_Algo_SetMaxIter (NM_Solv_Def.f90:198-207)
        if int(max_iter) < 1:
            raise ValueError("NM_Solver_Algo_SetMaxIter: Max iterations must be >= 1")
        self.max_iter = int(max_iter)


@dataclass
class NM_Solver_State:
    """NM_Solver_State (NM_Solv_Def.f90:105-117).  b and x are the right-hand
    side and solution (host numpy or CUDA tensors); x is the initial guess when
    use_x0 is set in the algo.  rnorm is ||b - K x|| / ||b|| in FP64."""
    niter: int = 0
    rnorm: float = 0.0
    dunorm: float = 0.0
    converged: bool = False
    initial_residual: float = 0.0
    solve_time: float = 0.0  # ms of device time
    convergence_flag: int = 0  # 0 ok, 2 max-iter, 3 breakdown / stall
    residual_history: np.ndarray | None = None
    x: object = None
    b: object = None
    n_refine: int = 0


@dataclass
class NM_Solver_Ctx:
    """NM_Solver_Ctx (NM_Solv_Def.f90:122-132): the hot-path work arrays; here
    the GPU context that owns them and the assembled matrix."""
    model: FemModel = None


def NM_Solver_PCG(desc: NM_Solver_Desc, state: NM_Solver_State, algo: NM_Solver_Algo,
                  ctx: NM_Solver_Ctx) -> ErrorStatusType:
    """NM_Solver_PCG (ufc_core/L2_NM/Solver/NM_Solv_Core.f90:363-423): PCG on
    the assembled stiffness of ctx.model for state%b, solution in state%x.
    Stops when the FP64 residual ||b - K x|| <= tolerance ||b||; returns
    IF_STATUS_NOT_CONVERGED after max_iter (the reference returns
    IF_STATUS_INVALID there, with the same message)."""
    m = ctx.model
    if desc.n and desc.n != m.n_dof:
        return ErrorStatusType(IF_STATUS_INVALID, f"desc%n = {desc.n} but the model has {m.n_dof} DOF",
                               "NM_Solver_PCG")
    if state.b is None:
        return ErrorStatusType(IF_STATUS_INVALID, "state%b is not associated", "NM_Solver_PCG")
    try:
        x, st = m.solve(state.b, algo, x=state.x, raise_on_not_converged=False)
    except UfcError as e:
        return ErrorStatusType(e.status_code, e.message, "NM_Solver_PCG")
    state.x = x
    state.niter, state.rnorm, state.converged = st.niter, st.rnorm, st.converged
    state.initial_residual, state.solve_time = st.initial_residual, st.solve_time
    state.convergence_flag, state.n_refine = st.convergence_flag, st.n_refine
    state.residual_history = m.residual_history()
    if not st.converged:
        return ErrorStatusType(IF_STATUS_NOT_CONVERGED, "[NM_Solver_PCG]: did not converge", "NM_Solver_PCG")
    return ErrorStatusType(IF_STATUS_OK, "", "NM_Solver_PCG")


# ---------------------------------------------------------------- L4 material and element
@dataclass
class PH_Mat_Update_Arg:
    """PH_Mat_Update_Arg (ufc_core/L4_PH/Material/PH_Mat_KernelDefn.f90:18-59),
    one row per integration point: mat_model_id 101 (elastic) or 201 (J2),
    props [E, nu] or [E, nu, sigma_y, H] (per point or shared), stress_n and
    dstrain in Voigt (xx, yy, zz, gxy, gyz, gzx), sdv_n = [epeq, eps_p(6)].
    Outputs: stress_new, sdv_tr, D_tang (consistent tangent), yielded."""
    mat_model_id: int
    props: np.ndarray
    stress_n: np.ndarray
    dstrain: np.ndarray
    sdv_n: np.ndarray | None = None
    stress_new: np.ndarray | None = None
    sdv_tr: np.ndarray | None = None
    D_tang: np.ndarray | None = None
    yielded: np.ndarray | None = None


def PH_Mat_UpdateStress(ctx: NM_Solver_Ctx, arg: PH_Mat_Update_Arg) -> ErrorStatusType:
    """UpdateStress / ComputeCTM of the material kernels
    (PH_Mat_KernelDefn.f90:18-59; J2: PH_J2_ComputeStress,
    PH_Mat_Plast_J2_Iso_Core.f90:133-207) for a batch of points on the GPU."""
    out, status = _run("PH_Mat_UpdateStress", ctx.model.mat_update_batch, arg.mat_model_id, arg.props,
                       arg.stress_n, arg.dstrain, arg.sdv_n)
    if out is not None:
        arg.stress_new, arg.sdv_tr, arg.D_tang, arg.yielded = out
    return status


@dataclass
class PH_Element_Compute_Fe_Arg:
    """PH_Element_Compute_Fe_Arg (ufc_core/L4_PH/Element/PH_Elem_Def.f90:343-355),
    batched over every element: u is the global displacement; Fe the assembled
    internal force, R = F_ext - F_int on the free DOFs."""
    u: object = None
    F_ext: object = None
    update_state: bool = False
    Fe: object = None
    R: object = None
    residual_norm: float = 0.0


def PH_Element_Compute_Ke(ctx: NM_Solver_Ctx, build=A.BUILD_FP64) -> ErrorStatusType:
    """Compute_Ke of every element with its scatter into the device CSR values
    (PH_Element_Compute_Ke_Arg, PH_Elem_Def.f90:331-341, called per element by
    RT_Asm_Solv.f90:1883,1946): one batched launch set per colour."""
    return _run("PH_Element_Compute_Ke", ctx.model.assemble, build)[1]


def PH_Element_Compute_Fe(ctx: NM_Solver_Ctx, arg: PH_Element_Compute_Fe_Arg) -> ErrorStatusType:
    """F_int = sum_e sum_gp w detJ B^T sigma for every element
    (PH_Elem_C3D8_IntForce, PH_Elem_C3D8.f90:734-757)."""
    out, status = _run("PH_Element_Compute_Fe", ctx.model.internal_force, arg.u, f_ext=arg.F_ext,
                       update_state=arg.update_state)
    if out is not None:
        arg.Fe, arg.R, arg.residual_norm, _ = out
    return status


# ---------------------------------------------------------------- L5 assembly and nonlinear driver
@dataclass
class RT_AsmColor_Result:
    """RT_AsmColor_Result (ufc_core/L5_RT/Assembly/RT_Asm_Color.f90:26-32), with
    the reference's 1-based colours and element ids."""
    color_of: np.ndarray | None = None     # [n_elem] colour of each element, 1..n_colors
    n_colors: int = 0
    color_count: np.ndarray | None = None  # [n_colors] elements per colour
    color_start: np.ndarray | None = None  # [n_colors + 1] first position of each colour in color_elems
    color_elems: np.ndarray | None = None  # [n_elem] element ids grouped by colour, ascending inside one


def color_groups(color_of: np.ndarray):
    """(n_colors, color_count, color_start, color_elems) of 1-based colours, in
    the order of build_color_groups (RT_Asm_Color.f90:148-180): a colour's
    elements in ascending id, all 1-based."""
    color_of = np.asarray(color_of, dtype=np.int32)
    n = int(color_of.max()) if color_of.size else 0
    count = np.bincount(color_of - 1, minlength=n).astype(np.int32)
    start = np.empty(n + 1, dtype=np.int32)
    start[0] = 1
    np.cumsum(count, out=start[1:])
    start[1:] += 1
    elems = (np.argsort(color_of, kind="stable") + 1).astype(np.int32)
    return n, count, start, elems


def RT_AsmColor_Build(ctx: NM_Solver_Ctx, result: RT_AsmColor_Result) -> ErrorStatusType:
    """RT_AsmColor_Build (RT_Asm_Color.f90:36-146): the greedy colouring of the
    model's elements (ascending order, smallest colour no element sharing a node
    already has), as ufc_pattern_build computed it on the device, with the
    colour groups."""
    colours, status = _run("RT_AsmColor_Build", ctx.model.colors, 1)
    if colours is not None:
        result.color_of = colours
        result.n_colors, result.color_count, result.color_start, result.color_elems = color_groups(colours)
    return status


def RT_Asm_GlobalStiffness(ctx: NM_Solver_Ctx, build=A.BUILD_FP64) -> ErrorStatusType:
    """RT_Asm_GlobalStiffness (ufc_core/L5_RT/Assembly/RT_Asm_Solv.f90:1762-1985):
    element loop and scatter into the CSR whose pattern the model built once."""
    return _run("RT_Asm_GlobalStiffness", ctx.model.assemble, build)[1]


def RT_Asm_ComputeResidual(ctx: NM_Solver_Ctx, u, F_ext):
    """RT_Asm_ComputeResidual (RT_Asm_Solv.f90:1311-1426): (R, status) with
    R = F_ext - F_int(u) on the free DOFs (zero on prescribed DOFs)."""
    out, status = _run("RT_Asm_ComputeResidual", ctx.model.internal_force, u, f_ext=F_ext, update_state=False)
    return (out[1] if out is not None else None), status


@dataclass
class MD_NonlinSolv:
    """The Newton-Raphson controls of MD_NonlinSolv read by
    RT_NLSolver_NewtonRaph (RT_Solv_Nonlin.f90:807-830): iteration limit, the
    force tolerance (||R_free|| <= tol max(||F_ext||, ||F_int||)) and the
    linear solver of each iteration."""
    max_iterations: int = 25
    tolerance_force: float = 1e-8
    linear: SolverAlgo = field(default_factory=SolverAlgo)


@dataclass
class MD_SolverState:
    """The fields of MD_SolverState an increment fills: iterations, convergence,
    the final residual norm and its history, the linear iterations spent."""
    iteration: int = 0
    converged: bool = False
    residual_norm: float = 0.0
    residual_history: list = field(default_factory=list)
    lin_iters_total: int = 0


def RT_NLSolver_NewtonRaph(solver: MD_NonlinSolv, state: MD_SolverState, ctx: NM_Solver_Ctx, u_prescribed,
                           F_ext=None):
    """RT_NLSolver_NewtonRaph (ufc_core/L5_RT/Solver/RT_Solv_Nonlin.f90:807-1002)
    for one increment, all on the device: return map, internal force,
    convergence test, consistent-tangent assembly and PCG per iteration, with
    the increment's prescribed values u_prescribed (one per Dirichlet DOF).
    Returns (result, status) as the reference's LOGICAL result and status; the
    trial state stays uncommitted (RT_Step_Commit_State: state_commit)."""
    out, status = _run("RT_NLSolver_NewtonRaph", ctx.model.nr_increment, u_prescribed, F_ext,
                       max_iterations=solver.max_iterations, tolerance_force=solver.tolerance_force,
                       lin=solver.linear)
    if out is None:
        return False, status
    state.iteration, state.converged = out.iterations, out.converged
    state.residual_norm, state.residual_history = out.residual_norm, out.res_hist
    state.lin_iters_total = out.lin_iters_total
    if not out.converged:
        status = ErrorStatusType(IF_STATUS_NOT_CONVERGED, "Newton-Raphson did not converge", "RT_NLSolver_NewtonRaph")
    return out.converged, status


def RT_StepDriver_Execute(ctx: NM_Solver_Ctx, solver: MD_NonlinSolv, u_prescribed_end=None, f_ext_end=None,
                          **step_ctl):
    """RT_StepDriver_Execute (ufc_core/L5_RT/StepDriver/RT_Step_Exec.f90:415-600):
    increments with commit, rollback and cutback under the RT_Step_Stp_Ctl_Algo
    controls given as keywords (time_period, dt_initial, dt_min, dt_max,
    max_increments, max_cutbacks, ...).  Returns (StepResult, status)."""
    out, status = _run("RT_StepDriver_Execute", ctx.model.nr_step, u_prescribed_end, f_ext_end,
                       max_iterations=solver.max_iterations, tolerance_force=solver.tolerance_force,
                       lin=solver.linear, **step_ctl)
    if out is not None and not out.completed:
        status = ErrorStatusType(IF_STATUS_NOT_CONVERGED, "step did not complete", "RT_StepDriver_Execute")
    return out, status
