"""Host-side model object over the C-ABI.

`FemModel` owns one `ufc_ctx` (device memory for mesh, pattern, matrix values,
solver vectors and material state) and exposes the hot path in the order the
reference's L5 runtime calls it:

    mesh/material/BC  ->  pattern_build (once)      RT_CSR_FromTripletMerged
    assemble                                        RT_Asm_GlobalStiffness
    internal_force / residual                       RT_Asm_ComputeResidual
    solve                                           NM_Solver_PCG / iter_pcg
    nr_increment, commit, rollback                  RT_NLSolver_NewtonRaph, RT_Step_Exec

Arrays may be numpy arrays (host) or torch tensors (host or CUDA); CUDA tensors
are passed by device pointer and used in order on torch's current stream.
Every failure raises `UfcError` carrying the reference's IF_STATUS_* code; the
library has no CPU fallback and loading fails loudly when it is not built.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

try:  # torch is optional for the host path but required for device tensors
    import torch
except Exception:  # pragma: no cover
    torch = None


class UfcError(RuntimeError):
    """A non-OK status from the library (ErrorStatusType, IF_Err_Def.f90:118-135)."""

    def __init__(self, status: int, message: str, where: str = ""):
        self.status_code = int(status)
        self.message = message
        name = A.STATUS_NAMES.get(self.status_code, str(self.status_code))
        super().__init__(f"[{where}] IF_STATUS_{name} ({self.status_code}): {message}")


def _is_torch(x):
    return torch is not None and isinstance(x, torch.Tensor)


class _Buf:
    """Pointer + memory space of a numpy array or torch tensor (kept alive)."""

    def __init__(self, x, dtype, count=None, writable=False):
        self.obj = None
        if x is None:
            self.ptr, self.mem = None, A.MEM_HOST
            return
        if _is_torch(x):
            tdt = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32}[dtype]
            if x.dtype != tdt or not x.is_contiguous():
                if writable:
                    raise TypeError(f"output tensor must be contiguous {tdt}")
                x = x.to(tdt).contiguous()
            self.obj = x
            self.ptr = x.data_ptr()
            self.mem = A.MEM_DEVICE if x.is_cuda else A.MEM_HOST
            n = x.numel()
        else:
            if writable:
                if not (isinstance(x, np.ndarray) and x.dtype == dtype and x.flags.c_contiguous):
                    raise TypeError(f"output array must be C-contiguous {np.dtype(dtype)}")
                arr = x
            else:
                arr = np.ascontiguousarray(x, dtype=dtype)
            self.obj = arr
            self.ptr = arr.ctypes.data
            self.mem = A.MEM_HOST
            n = arr.size
        if count is not None and n < count:
            raise ValueError(f"array has {n} entries, {count} needed")


def _same_mem(*bufs):
    mems = {b.mem for b in bufs if b.ptr is not None}
    if len(mems) > 1:
        raise ValueError("mix of host and device arrays in one call")
    return mems.pop() if mems else A.MEM_HOST


@dataclass
class SolverAlgo:
    """NM_Solver_Algo (ufc_core/L2_NM/Solver/NM_Solv_Def.f90:86-100)."""

    method: int = A.SOLV_METHOD_CG
    precond_type: int = A.SOLV_PREC_JACOBI
    max_iter: int = 100000
    tolerance: float = 1e-10
    abs_tolerance: float = 0.0
    precision_mode: int = A.PRECISION_FP64
    refine_delta: float = 0.0
    check_every: int = 0
    use_x0: int = 0
    refine_policy: int = A.REFINE_KEEP_DIRECTION
    accumulate: int = A.ACCUMULATE_STORAGE

    def to_c(self):
        return A.SolverAlgo(self.method, self.precond_type, self.max_iter, self.precision_mode, self.tolerance,
                            self.abs_tolerance, self.refine_delta, self.check_every, self.use_x0,
                            self.refine_policy, self.accumulate)


@dataclass
class SolverState:
    """NM_Solver_State (ufc_core/L2_NM/Solver/NM_Solv_Def.f90:105-117)."""

    niter: int = 0
    n_refine: int = 0
    converged: bool = False
    convergence_flag: int = 0
    rnorm: float = 0.0
    initial_residual: float = 0.0
    solve_time: float = 0.0  # ms
    status: int = 0
    fp64_iters: int = 0

    @classmethod
    def from_c(cls, s, status=0):
        return cls(s.niter, s.n_refine, bool(s.converged), s.convergence_flag, s.rnorm, s.initial_residual,
                   s.solve_time, status, s.fp64_iters)


@dataclass
class StepResult:
    """Outcome of FemModel.nr_step; history rows are (step time, dt, Newton
    iterations, converged) per attempted increment."""
    completed: bool
    final_time: float
    increments: int
    cutbacks: int
    attempts: int
    nr_iterations: int
    lin_iters_total: int
    history: list = field(default_factory=list)
    status: int = 0


@dataclass
class NrResult:
    iterations: int
    converged: bool
    lin_iters_total: int
    residual_norm: float
    res_hist: list = field(default_factory=list)


class FemModel:
    """One C3D8 model on one GPU (one `ufc_ctx`)."""

    def __init__(self, device: int = 0, stream=None, lib=None):
        self.lib = lib or A.load()
        h = C.c_void_p()
        st = self.lib.ufc_ctx_create(int(device), C.byref(h))
        if st != 0:
            raise UfcError(st, "ufc_ctx_create failed (no sm_100 GPU or out of memory)", "ufc_ctx_create")
        self.h = h
        self.device = device
        self.n_nodes = self.n_elems = self.n_dof = 0
        self.info = None
        self.fixed = np.zeros(0, dtype=np.int32)
        self.assembled = 0
        self._moduli_key = None
        if stream is None and torch is not None and torch.cuda.is_available():
            stream = torch.cuda.current_stream(device)
        if stream is not None:
            self.set_stream(stream)

    # ---------------------------------------------------------------- plumbing
    def _check(self, st, where):
        if st != 0:
            buf = C.create_string_buffer(512)
            self.lib.ufc_last_error(self.h, buf, 512)
            raise UfcError(st, buf.value.decode(errors="replace"), where)
        return st

    def set_stream(self, stream):
        ptr = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream or 0)
        self._check(self.lib.ufc_ctx_set_stream(self.h, C.c_void_p(ptr)), "ufc_ctx_set_stream")

    def close(self):
        if getattr(self, "h", None):
            self.lib.ufc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- set-up
    def set_mesh(self, coords, conn, index_base=0):
        cb = _Buf(coords, np.float64)
        kb = _Buf(conn, np.int32)
        mem = _same_mem(cb, kb)
        n_nodes = int(np.prod(np.shape(coords))) // 3
        n_elems = int(np.prod(np.shape(conn))) // 8
        d = A.MeshDesc(n_nodes, n_elems, cb.ptr, kb.ptr, index_base, mem)
        self._check(self.lib.ufc_mesh_set(self.h, C.byref(d)), "ufc_mesh_set")
        self.n_nodes, self.n_elems, self.n_dof = n_nodes, n_elems, 3 * n_nodes
        self.assembled = 0

    def set_material(self, mat_model_id, props, per_element=None):
        pb = _Buf(props, np.float64)
        shape = np.shape(props)
        if per_element is None:
            per_element = len(shape) == 2
        nprops = shape[-1]
        d = A.MaterialDesc(int(mat_model_id), int(nprops), int(per_element), pb.ptr, pb.mem)
        self._check(self.lib.ufc_material_set(self.h, C.byref(d)), "ufc_material_set")
        self.mat_model_id = int(mat_model_id)
        self.assembled = 0

    def set_bc(self, dofs, values=None):
        dofs = np.ascontiguousarray(dofs, dtype=np.int32)
        vb = _Buf(values, np.float64)
        d = A.BcDesc(int(dofs.size), dofs.ctypes.data, vb.ptr, A.MEM_HOST)
        self._check(self.lib.ufc_bc_set(self.h, C.byref(d)), "ufc_bc_set")
        self.fixed = dofs
        self.assembled = 0

    def pattern_build(self):
        info = A.PatternInfo()
        self._check(self.lib.ufc_pattern_build(self.h, C.byref(info)), "ufc_pattern_build")
        self.info = info
        return {"n_dof": info.n_dof, "nnz": info.nnz, "nnzb": info.nnzb, "sell_blocks": info.sell_blocks,
                "n_colors": info.n_colors, "max_row_blocks": info.max_row_blocks}

    def colors(self, index_base=0):
        """Element colours of the pattern build (RT_AsmColorResult%color_of of
        RT_AsmColor_Build), int32 on the host."""
        out = np.zeros(self.n_elems, dtype=np.int32)
        self._check(self.lib.ufc_pattern_colors(self.h, out.ctypes.data, int(index_base), A.MEM_HOST),
                    "ufc_pattern_colors")
        return out

    @classmethod
    def from_problem(cls, p, device=0, build_pattern=True, lib=None):
        """Model of a `mesh.Problem` (mesh, material, Dirichlet set)."""
        m = cls(device, lib=lib)
        m.set_mesh(p.coords, p.conn)
        m.set_material(p.mat_model_id, p.props)
        m.set_bc(p.fixed, p.fixed_values)
        if build_pattern:
            m.pattern_build()
        m.problem = p
        return m

    # ---------------------------------------------------------------- element
    def assemble(self, build=A.BUILD_FP64):
        a = A.ElemKeArg(int(build), 0, 0.0)
        self._check(self.lib.ufc_elem_compute_ke(self.h, C.byref(a)), "ufc_elem_compute_ke")
        self.assembled |= int(build)
        return a.elapsed_ms

    def internal_force(self, u, f_ext=None, want_r=True, update_state=True):
        """(F_int, R = f_ext - F_int on free DOFs, ||R||, ||F_int||)."""
        like = u
        ub = _Buf(u, np.float64, self.n_dof)
        fb = _Buf(f_ext, np.float64, self.n_dof)
        mem = _same_mem(ub, fb)
        fint = self._empty(self.n_dof, np.float64, like)
        r = self._empty(self.n_dof, np.float64, like) if want_r else None
        fib, rb = _Buf(fint, np.float64, writable=True), _Buf(r, np.float64, writable=True)
        a = A.ElemFeArg(ub.ptr, fb.ptr, fib.ptr, rb.ptr, mem, int(update_state), 0.0, 0.0, 0)
        self._check(self.lib.ufc_elem_compute_fint(self.h, C.byref(a)), "ufc_elem_compute_fint")
        return fint, r, a.rnorm, a.fint_norm

    def stress(self, u=None, want_sigma=True):
        like = u if u is not None else np.zeros(1)
        G = 8 * self.n_elems
        sig = self._empty(G * 6, np.float64, like) if want_sigma else None
        vm = self._empty(G, np.float64, like)
        ub = _Buf(u, np.float64)
        sb, vb = _Buf(sig, np.float64, writable=True), _Buf(vm, np.float64, writable=True)
        mem = _same_mem(ub, sb, vb)
        self._check(self.lib.ufc_stress_eval(self.h, ub.ptr, sb.ptr, vb.ptr, mem), "ufc_stress_eval")
        return (sig.reshape(self.n_elems, 8, 6) if sig is not None else None), vm.reshape(self.n_elems, 8)

    def mat_update_batch(self, mat_model_id, props, stress_n, dstrain, sdv_n=None):
        """Material-point batch (PH_Mat_Update_Arg rows); returns (stress, sdv, ddsdde, yielded)."""
        stress_n = np.ascontiguousarray(stress_n, dtype=np.float64).reshape(-1, 6)
        n = stress_n.shape[0]
        props = np.ascontiguousarray(props, dtype=np.float64)
        per_point = int(props.ndim == 2)
        nprops = props.shape[-1]
        de = np.ascontiguousarray(dstrain, dtype=np.float64).reshape(n, 6)
        sv = None if sdv_n is None else np.ascontiguousarray(sdv_n, dtype=np.float64).reshape(n, 7)
        s = np.zeros((n, 6))
        v = np.zeros((n, 7))
        D = np.zeros((n, 36))
        y = np.zeros(n, dtype=np.int32)
        a = A.MatUpdateArg(int(mat_model_id), n, nprops, per_point, props.ctypes.data, stress_n.ctypes.data,
                           de.ctypes.data, None if sv is None else sv.ctypes.data, s.ctypes.data, v.ctypes.data,
                           D.ctypes.data, y.ctypes.data, A.MEM_HOST, 0)
        self._check(self.lib.ufc_mat_update_batch(self.h, C.byref(a)), "ufc_mat_update_batch")
        return s, v, D.reshape(n, 6, 6), y.astype(bool)

    # ---------------------------------------------------------------- matrix
    def csr_export(self, index_base=0, values=True, values32=False):
        """Canonical CSR (row_ptr int64, col int32, values float64/float32) on the host."""
        n, nnz = self.info.n_dof, self.info.nnz
        rp = np.zeros(n + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int32)
        v = np.zeros(nnz) if values else None
        v32 = np.zeros(nnz, dtype=np.float32) if values32 else None
        a = A.CsrExportArg(index_base, A.MEM_HOST, rp.ctypes.data, col.ctypes.data,
                           None if v is None else v.ctypes.data, None if v32 is None else v32.ctypes.data)
        self._check(self.lib.ufc_csr_export(self.h, C.byref(a)), "ufc_csr_export")
        return rp, col, v if values else v32, v32

    def spmv(self, x, precision=A.PRECISION_FP64, out=None):
        dt = np.float64 if precision == A.PRECISION_FP64 else np.float32
        y = out if out is not None else self._empty(self.n_dof, dt, x)
        xb, yb = _Buf(x, dt, self.n_dof), _Buf(y, dt, self.n_dof, writable=True)
        self._check(self.lib.ufc_spmv(self.h, int(precision), xb.ptr, yb.ptr, _same_mem(xb, yb)), "ufc_spmv")
        return y

    # ---------------------------------------------------------------- solver
    def solve(self, b, algo: SolverAlgo | None = None, x=None, raise_on_not_converged=True):
        """Jacobi-PCG on the eliminated system; returns (x, SolverState)."""
        algo = algo or SolverAlgo()
        if x is None:
            x = self._empty(self.n_dof, np.float64, b)
        bb, xb = _Buf(b, np.float64, self.n_dof), _Buf(x, np.float64, self.n_dof, writable=True)
        ca = algo.to_c()
        cs = A.SolverState()
        st = self.lib.ufc_pcg_solve(self.h, bb.ptr, xb.ptr, _same_mem(bb, xb), C.byref(ca), C.byref(cs))
        if st != 0 and not (st == A.STATUS_NOT_CONVERGED and not raise_on_not_converged):
            self._check(st, "ufc_pcg_solve")
        return x, SolverState.from_c(cs, st)

    def solve_block(self, B, algo: SolverAlgo | None = None, X=None, raise_on_not_converged=True):
        """nrhs independent solves sharing each SpMV; B is [nrhs, n_dof]."""
        algo = algo or SolverAlgo()
        nrhs = int(B.shape[0])
        if X is None:
            X = self._empty(nrhs * self.n_dof, np.float64, B).reshape(nrhs, self.n_dof)
        bb, xb = _Buf(B, np.float64, nrhs * self.n_dof), _Buf(X, np.float64, nrhs * self.n_dof, writable=True)
        ca = algo.to_c()
        cs = (A.SolverState * nrhs)()
        st = self.lib.ufc_pcg_solve_block(self.h, nrhs, bb.ptr, xb.ptr, _same_mem(bb, xb), C.byref(ca), cs)
        if st != 0 and not (st == A.STATUS_NOT_CONVERGED and not raise_on_not_converged):
            self._check(st, "ufc_pcg_solve_block")
        return X, [SolverState.from_c(s, st) for s in cs]

    # ---------------------------------------------------------------- multigrid
    def mg_setup(self, nx, ny, nz, max_levels=0, degree=0, ratio=0.0, coarse_max=0, precision=A.PRECISION_FP64):
        """Geometric multigrid hierarchy of the nx x ny x nz box (ufc_mg_setup);
        solve with SolverAlgo(precond_type=SOLV_PREC_MG).  precision
        PRECISION_FP32_REFINE runs the cycle in FP32.  Returns (levels,
        coarsest DOF, set-up ms)."""
        a = A.MgArg()
        a.nx, a.ny, a.nz, a.max_levels, a.degree = int(nx), int(ny), int(nz), int(max_levels), int(degree)
        a.ratio, a.coarse_max, a.precision = float(ratio), int(coarse_max), int(precision)
        self._check(self.lib.ufc_mg_setup(self.h, C.byref(a)), "ufc_mg_setup")
        return a.levels, a.coarse_dof, a.setup_ms

    def mg_apply(self, r, out=None):
        """z = M r, one V-cycle."""
        z = out if out is not None else self._empty(self.n_dof, np.float64, r)
        rb, zb = _Buf(r, np.float64, self.n_dof), _Buf(z, np.float64, self.n_dof, writable=True)
        self._check(self.lib.ufc_mg_apply(self.h, rb.ptr, zb.ptr, _same_mem(rb, zb)), "ufc_mg_apply")
        return z

    def mg_export(self, level):
        """Canonical CSR (row_ptr, col, values) of the operator of one multigrid level."""
        n, nnz = C.c_int64(0), C.c_int64(0)
        self._check(self.lib.ufc_mg_level_info(self.h, int(level), C.byref(n), C.byref(nnz)), "ufc_mg_level_info")
        rp = np.zeros(n.value + 1, dtype=np.int64)
        col = np.zeros(nnz.value, dtype=np.int32)
        v = np.zeros(nnz.value)
        a = A.CsrExportArg(0, A.MEM_HOST, rp.ctypes.data, col.ctypes.data, v.ctypes.data, None)
        self._check(self.lib.ufc_mg_export(self.h, int(level), C.byref(a)), "ufc_mg_export")
        return rp, col, v

    def set_instrument(self, on=True):
        self._check(self.lib.ufc_ctx_set_instrument(self.h, int(on)), "ufc_ctx_set_instrument")

    def last_timing(self):
        t = A.TimingInfo()
        self._check(self.lib.ufc_last_timing(self.h, C.byref(t)), "ufc_last_timing")
        return {"spmv_launches": t.spmv_launches, "spmv_ms": t.spmv_ms, "spmv_bytes": t.spmv_bytes,
                "precision": t.precision, "kernel_launches": t.kernel_launches}

    def residual_history(self, max_len=1 << 20):
        """||r_k||_2 of the CG recurrence per iteration of the last solve."""
        out = np.zeros(max_len)
        n = C.c_int32(0)
        self._check(self.lib.ufc_last_residual_history(self.h, out.ctypes.data, int(max_len), C.byref(n)),
                    "ufc_last_residual_history")
        return out[: n.value].copy()

    # ---------------------------------------------------------------- nonlinear
    def nr_increment(self, u_prescribed, f_ext=None, max_iterations=25, tolerance_force=1e-8,
                     lin: SolverAlgo | None = None):
        lin = lin or SolverAlgo()
        ub = _Buf(u_prescribed, np.float64)
        fb = _Buf(f_ext, np.float64)
        a = A.NrArg()
        a.u_prescribed = ub.ptr
        a.f_ext = fb.ptr
        a.mem = _same_mem(ub, fb)
        a.max_iterations = int(max_iterations)
        a.tolerance_force = float(tolerance_force)
        a.lin = lin.to_c()
        st = self.lib.ufc_nr_increment(self.h, C.byref(a))
        res = NrResult(a.iterations, bool(a.converged), a.lin_iters_total, a.residual_norm,
                       list(a.res_hist[: max(a.iterations + 1, 1)]))
        self._check(st, "ufc_nr_increment")
        return res

    def nr_step(self, u_prescribed_end=None, f_ext_end=None, f_ext_start=None, time_period=1.0, dt_initial=1.0,
                dt_min=1e-5, dt_max=1.0, max_increments=100, max_cutbacks=5, auto_dt=True, target_iters=6,
                growth_threshold=0.8, growth_factor=1.25, cutback_factor=0.5, max_iterations=25,
                tolerance_force=1e-8, lin: SolverAlgo | None = None, raise_on_failure=False):
        """One step with automatic increments and cutbacks (ufc_nr_step); the
        defaults are the reference's RT_Step_Stp_Ctl_Algo values."""
        lin = lin or SolverAlgo()
        ub = _Buf(u_prescribed_end, np.float64, self.fixed.size if u_prescribed_end is not None else None)
        fsb = _Buf(f_ext_start, np.float64, self.n_dof if f_ext_start is not None else None)
        feb = _Buf(f_ext_end, np.float64, self.n_dof if f_ext_end is not None else None)
        cap = int(max_increments)
        ht, hd = np.zeros(cap), np.zeros(cap)
        hi, hc = np.zeros(cap, dtype=np.int32), np.zeros(cap, dtype=np.int32)
        a = A.StepArg()
        a.u_prescribed_end, a.f_ext_start, a.f_ext_end = ub.ptr, fsb.ptr, feb.ptr
        a.mem = _same_mem(ub, fsb, feb)
        a.time_period, a.dt_initial, a.dt_min, a.dt_max = time_period, dt_initial, dt_min, dt_max
        a.max_increments, a.max_cutbacks, a.auto_dt, a.target_iters = cap, max_cutbacks, int(auto_dt), target_iters
        a.growth_threshold, a.growth_factor, a.cutback_factor = growth_threshold, growth_factor, cutback_factor
        a.max_iterations, a.tolerance_force, a.lin = max_iterations, tolerance_force, lin.to_c()
        a.hist_time, a.hist_dt = ht.ctypes.data, hd.ctypes.data
        a.hist_iters, a.hist_converged = hi.ctypes.data, hc.ctypes.data
        a.hist_cap = cap
        st = self.lib.ufc_nr_step(self.h, C.byref(a))
        k = min(a.attempts, cap)
        res = StepResult(bool(a.completed), a.final_time, a.increments, a.cutbacks, a.attempts, a.nr_iterations,
                         a.lin_iters_total, [(float(ht[i]), float(hd[i]), int(hi[i]), bool(hc[i])) for i in range(k)],
                         st)
        if st != A.STATUS_NOT_CONVERGED or raise_on_failure:
            self._check(st, "ufc_nr_step")
        return res

    def load_faces(self, elem, face, traction=None, pressure=None, index_base=0, out=None):
        """Equivalent nodal forces of face tractions ([n_faces, 3]) and/or
        pressures ([n_faces]) on the faces `face` (1..6) of elements `elem`."""
        like = traction if traction is not None else (pressure if pressure is not None else elem)
        n_faces = len(elem)
        f = out if out is not None else self._empty(self.n_dof, np.float64, like if _is_torch(like) else np.zeros(1))
        eb, fb = _Buf(elem, np.int32, n_faces), _Buf(face, np.int32, n_faces)
        tb = _Buf(traction, np.float64, 3 * n_faces if traction is not None else None)
        pb = _Buf(pressure, np.float64, n_faces if pressure is not None else None)
        ob = _Buf(f, np.float64, self.n_dof, writable=True)
        a = A.FaceLoadArg(n_faces, eb.ptr, fb.ptr, tb.ptr, pb.ptr, int(index_base), _same_mem(eb, fb, tb, pb, ob),
                          ob.ptr)
        self._check(self.lib.ufc_load_faces(self.h, C.byref(a)), "ufc_load_faces")
        return f

    def stress_nodal(self, u=None, want_sigma=True):
        """Nodal stress [n_nodes, 6] (extrapolated from the Gauss points and
        averaged over elements) and its von Mises value [n_nodes]."""
        like = u if u is not None else np.zeros(1)
        sig = self._empty(self.n_nodes * 6, np.float64, like) if want_sigma else None
        vm = self._empty(self.n_nodes, np.float64, like)
        ub = _Buf(u, np.float64, self.n_dof if u is not None else None)
        sb, vb = _Buf(sig, np.float64, writable=True), _Buf(vm, np.float64, writable=True)
        self._check(self.lib.ufc_stress_nodal(self.h, ub.ptr, sb.ptr, vb.ptr, _same_mem(ub, sb, vb)),
                    "ufc_stress_nodal")
        return (sig.reshape(self.n_nodes, 6) if sig is not None else None), vm

    def reactions(self, u=None, f_ext=None):
        """RF = F_int(u) - F_ext at the prescribed DOFs, in the order of set_bc."""
        like = u if u is not None else (f_ext if f_ext is not None else np.zeros(1))
        rf = self._empty(max(self.fixed.size, 1), np.float64, like)
        ub = _Buf(u, np.float64, self.n_dof if u is not None else None)
        fb = _Buf(f_ext, np.float64, self.n_dof if f_ext is not None else None)
        rb = _Buf(rf, np.float64, writable=True)
        self._check(self.lib.ufc_reactions(self.h, ub.ptr, fb.ptr, rb.ptr, _same_mem(ub, fb, rb)), "ufc_reactions")
        return rf[: self.fixed.size]

    def commit(self):
        self._check(self.lib.ufc_state_commit(self.h), "ufc_state_commit")

    def rollback(self):
        self._check(self.lib.ufc_state_rollback(self.h), "ufc_state_rollback")

    def displacement(self, out=None):
        u = out if out is not None else np.zeros(self.n_dof)
        b = _Buf(u, np.float64, self.n_dof, writable=True)
        self._check(self.lib.ufc_get_displacement(self.h, b.ptr, b.mem), "ufc_get_displacement")
        return u

    def set_displacement(self, u):
        b = _Buf(u, np.float64, self.n_dof)
        self._check(self.lib.ufc_set_displacement(self.h, b.ptr, b.mem), "ufc_set_displacement")

    def j2_state(self):
        G = 8 * self.n_elems
        epeq, sig, epl = np.zeros(G), np.zeros(G * 6), np.zeros(G * 6)
        self._check(self.lib.ufc_get_state(self.h, epeq.ctypes.data, sig.ctypes.data, epl.ctypes.data, A.MEM_HOST),
                    "ufc_get_state")
        return epeq.reshape(-1, 8), sig.reshape(-1, 8, 6), epl.reshape(-1, 8, 6)

    # ---------------------------------------------------------------- adjoint
    def adjoint_sensitivity(self, U, Lam):
        """dJ/dE_e = -sum_k lambda_k,e^T (Ke/E_e) u_k,e (U, Lam: [nrhs, n_dof])."""
        nrhs = 1 if len(U.shape) == 1 else int(U.shape[0])
        g = self._empty(self.n_elems, np.float64, U)
        ub, lb = _Buf(U, np.float64, nrhs * self.n_dof), _Buf(Lam, np.float64, nrhs * self.n_dof)
        gb = _Buf(g, np.float64, self.n_elems, writable=True)
        self._check(self.lib.ufc_adjoint_sensitivity(self.h, nrhs, ub.ptr, lb.ptr, gb.ptr, _same_mem(ub, lb, gb)),
                    "ufc_adjoint_sensitivity")
        return g

    # ---------------------------------------------------------------- helpers
    @staticmethod
    def _empty(n, dtype, like):
        if _is_torch(like):
            tdt = {np.float64: torch.float64, np.float32: torch.float32}[dtype]
            return torch.empty(n, dtype=tdt, device=like.device)
        return np.zeros(n, dtype=dtype)


def lifted_rhs(model: FemModel, f, fixed_values=None):
    """Right-hand side of the eliminated system: b_free = f - K_fc u_c,
    b_fixed = u_c (in place of the penalty of RT_Asm_ApplyBC_Displacement_Penalty,
    ufc_core/L5_RT/Assembly/RT_Asm_Solv.f90:427-483).  K_fc u_c is the free part
    of the internal force of the prescribed field alone."""
    p_fixed = model.fixed
    if _is_torch(f):
        b = f.clone()
        vals = torch.zeros(p_fixed.size, dtype=torch.float64, device=f.device) if fixed_values is None else \
            torch.as_tensor(fixed_values, dtype=torch.float64, device=f.device)
        idx = torch.as_tensor(p_fixed, dtype=torch.long, device=f.device)
        if bool((vals != 0).any()):
            uc = torch.zeros_like(f)
            uc[idx] = vals
            fint, _, _, _ = model.internal_force(uc, want_r=False, update_state=False)
            b -= fint
        b[idx] = vals
        return b
    b = np.array(f, dtype=np.float64)
    vals = np.zeros(p_fixed.size) if fixed_values is None else np.asarray(fixed_values, np.float64)
    if np.any(vals != 0):
        uc = np.zeros_like(b)
        uc[p_fixed] = vals
        fint, _, _, _ = model.internal_force(uc, want_r=False, update_state=False)
        b -= fint
    b[p_fixed] = vals
    return b
