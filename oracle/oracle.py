"""Python front end of the CPU FP64 oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.  The product path never imports it.

It wraps ``liborc.so`` (built from ufc_oracle.c by this folder's Makefile) and
adds the small drivers that the reference keeps in L5: the linear static solve
(RT_Asm_GlobalStiffness -> iter_pcg, ufc_core/L5_RT/Assembly/RT_Asm_Solv.f90:1762
and ufc_core/L2_NM/Solver/LinSolv/NM_Solv_IterSolver.f90:713) and the
Newton-Raphson increment (RT_NLSolver_NewtonRaph,
ufc_core/L5_RT/Solver/RT_Solv_Nonlin.f90:807-1002).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_c3d8_ke.argtypes = [_d, _d, C.c_void_p, _d]
        L.orc_j2_update.argtypes = [_d, _d, _d, C.c_double, _d, _d, C.POINTER(C.c_double), _d, _d]
        L.orc_csr_pattern.argtypes = [C.c_int32, C.c_int32, _i32, _i64, C.c_void_p]
        L.orc_csr_pattern.restype = C.c_int64
        L.orc_color_elements.argtypes = [C.c_int32, C.c_int32, _i32, _i32]
        L.orc_assemble.argtypes = [C.c_int32, C.c_int32, _d, _i32, _d, C.c_int32, C.c_void_p, _u8, _i32, C.c_int,
                                   _i64, _i32, _d]
        L.orc_spmv.argtypes = [C.c_int64, _i64, _i32, _d, _d, _d]
        L.orc_pcg.argtypes = [C.c_int64, _i64, _i32, _d, _d, _d, C.c_double, C.c_double, C.c_int,
                              C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_pcg_marked.argtypes = [C.c_int64, _i64, _i32, _d, _d, _d, C.c_double, C.c_int, C.c_double, _d,
                                     C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                     C.POINTER(C.c_double)]
        L.orc_fint.argtypes = [C.c_int32, C.c_int32, _d, _i32, _d, C.c_int32, C.c_int, _d, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _i32, C.c_int,
                               _d]
        L.orc_elastic_stress.argtypes = [C.c_int32, _d, _i32, _d, C.c_int32, _d, C.c_void_p, _d]
        L.orc_adjoint_dJdE.argtypes = [C.c_int32, C.c_int32, _d, _i32, _d, C.c_int32, C.c_int, _d, _d, _d]
        L.orc_hex8_grad.argtypes = [_d, _d, _d]
        L.orc_hex8_grad.restype = C.c_double
        L.orc_von_mises.argtypes = [_d]
        L.orc_von_mises.restype = C.c_double
        L.orc_num_threads.restype = C.c_int
        L.orc_set_threads.argtypes = [C.c_int]
        _LIB = L
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def num_threads():
    return lib().orc_num_threads()


def set_threads(n):
    lib().orc_set_threads(int(n))


# ---------------------------------------------------------------- pointwise


def iso_D(E, nu):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    return D


def c3d8_ke(X, D=None, Dgp=None):
    """24x24 element stiffness of one hex (X [8,3])."""
    Ke = np.zeros(576)
    D = np.ascontiguousarray(D if D is not None else np.zeros((6, 6)), dtype=np.float64).ravel()
    Dg = None if Dgp is None else np.ascontiguousarray(Dgp, dtype=np.float64).ravel()
    st = lib().orc_c3d8_ke(np.ascontiguousarray(X, dtype=np.float64).ravel(), D, _ptr(Dg), Ke)
    if st != 0:
        raise ValueError("non-positive Jacobian")
    return Ke.reshape(24, 24)


def j2_update(props, deps, sig_n=None, epeq_n=0.0, epl_n=None):
    """One J2 material-point update; returns (sigma, epeq, eps_p, D_ep, yielded)."""
    sig = np.zeros(6)
    epl = np.zeros(6)
    Dep = np.zeros(36)
    epeq = C.c_double(0.0)
    y = lib().orc_j2_update(np.asarray(props, np.float64), np.asarray(deps, np.float64),
                            np.zeros(6) if sig_n is None else np.asarray(sig_n, np.float64), float(epeq_n),
                            np.zeros(6) if epl_n is None else np.asarray(epl_n, np.float64), sig, C.byref(epeq),
                            epl, Dep)
    return sig, epeq.value, epl, Dep.reshape(6, 6), bool(y)


def von_mises(s):
    return lib().orc_von_mises(np.ascontiguousarray(s, dtype=np.float64))


# ---------------------------------------------------------------- global


@dataclass
class CSR:
    n: int
    row_ptr: np.ndarray  # int64 [n+1], 0-based
    col: np.ndarray  # int32 [nnz]
    val: np.ndarray  # float64 [nnz]

    def matvec(self, x):
        y = np.empty(self.n)
        lib().orc_spmv(self.n, self.row_ptr, self.col, self.val, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def to_dense(self):
        A = np.zeros((self.n, self.n))
        rows = np.repeat(np.arange(self.n), np.diff(self.row_ptr))
        A[rows, self.col] = self.val
        return A


def csr_pattern(n_nodes, conn):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    rp = np.zeros(3 * n_nodes + 1, dtype=np.int64)
    nnz = lib().orc_csr_pattern(n_nodes, conn.shape[0], conn, rp, None)
    if nnz < 0:
        raise ValueError("node valence above 64")
    col = np.zeros(nnz, dtype=np.int32)
    lib().orc_csr_pattern(n_nodes, conn.shape[0], conn, rp, _ptr(col))
    return rp, col


def color_elements(n_nodes, conn):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    color = np.zeros(conn.shape[0], dtype=np.int32)
    ncol = lib().orc_color_elements(n_nodes, conn.shape[0], conn, color)
    return color, ncol


class Model:
    """Mesh + pattern + colouring of one problem, reused across assemblies."""

    def __init__(self, p):
        self.p = p
        self.coords = np.ascontiguousarray(p.coords, dtype=np.float64)
        self.conn = np.ascontiguousarray(p.conn, dtype=np.int32)
        self.props = np.ascontiguousarray(p.props, dtype=np.float64)
        self.N, self.E = p.n_nodes, p.n_elems
        self.n = 3 * self.N
        self.row_ptr, self.col = csr_pattern(self.N, self.conn)
        self.color, self.ncol = color_elements(self.N, self.conn)
        self.fixed = np.zeros(self.n, dtype=np.uint8)
        self.fixed[p.fixed] = 1

    def assemble(self, Dgp=None, props=None, eliminate=True):
        """Stiffness with the Dirichlet rows/columns eliminated, or the full
        (singular) one when eliminate is False."""
        props = self.props if props is None else np.ascontiguousarray(props, dtype=np.float64)
        val = np.zeros(self.col.size)
        Dg = None if Dgp is None else np.ascontiguousarray(Dgp, dtype=np.float64)
        fixed = self.fixed if eliminate else np.zeros_like(self.fixed)
        st = lib().orc_assemble(self.N, self.E, self.coords, self.conn, props, props.shape[1], _ptr(Dg), fixed,
                                self.color, self.ncol, self.row_ptr, self.col, val)
        if st != 0:
            raise ValueError("non-positive Jacobian")
        return CSR(self.n, self.row_ptr, self.col, val)

    def fint_elastic(self, u, props=None):
        props = self.props if props is None else np.ascontiguousarray(props, dtype=np.float64)
        out = np.zeros(self.n)
        lib().orc_fint(self.N, self.E, self.coords, self.conn, props, props.shape[1], 0,
                       np.ascontiguousarray(u, dtype=np.float64), None, None, None, None, None, None, None, None,
                       self.color, self.ncol, out)
        return out

    def fint_j2(self, u, u_n, state):
        """J2 internal force at u from the committed state; returns (fint, trial)."""
        G = self.E * 8
        trial = {"sig": np.zeros(G * 6), "epeq": np.zeros(G), "epl": np.zeros(G * 6), "D": np.zeros(G * 36)}
        out = np.zeros(self.n)
        lib().orc_fint(self.N, self.E, self.coords, self.conn, self.props, self.props.shape[1], 1,
                       np.ascontiguousarray(u, dtype=np.float64), _ptr(np.ascontiguousarray(u_n, dtype=np.float64)),
                       _ptr(state["sig"]), _ptr(state["epeq"]), _ptr(state["epl"]), _ptr(trial["sig"]),
                       _ptr(trial["epeq"]), _ptr(trial["epl"]), _ptr(trial["D"]), self.color, self.ncol, out)
        return out, trial

    def lifted_rhs(self, f=None, fixed_values=None):
        """Right-hand side of the eliminated system: b_free = f - K_fc u_c and
        b_fixed = u_c (symmetric elimination in place of the reference's
        penalty, RT_Asm_Solv.f90:427-483)."""
        p = self.p
        f = p.f if f is None else f
        vals = p.fixed_values if fixed_values is None else fixed_values
        uc = np.zeros(self.n)
        uc[p.fixed] = vals
        b = np.array(f, dtype=np.float64)
        if np.any(vals != 0.0):
            b -= self.fint_elastic(uc)
        b[p.fixed] = vals
        return b

    def solve_linear(self, rtol=1e-10, max_iter=100000, f=None, K=None):
        K = self.assemble() if K is None else K
        b = self.lifted_rhs(f)
        x = np.zeros(self.n)
        it = C.c_int(0)
        rf = C.c_double(0.0)
        ri = C.c_double(0.0)
        st = lib().orc_pcg(self.n, K.row_ptr, K.col, K.val, b, x, rtol, 0.0, max_iter, C.byref(it), C.byref(rf),
                           C.byref(ri))
        return x, {"status": st, "iters": it.value, "res_final": rf.value, "res_init": ri.value, "K": K, "b": b}

    def elastic_vm(self, u, props=None):
        props = self.props if props is None else np.ascontiguousarray(props, dtype=np.float64)
        vm = np.zeros(self.E * 8)
        sig = np.zeros(self.E * 48)
        lib().orc_elastic_stress(self.E, self.coords, self.conn, props, props.shape[1],
                                 np.ascontiguousarray(u, dtype=np.float64), _ptr(sig), vm)
        return sig.reshape(self.E, 8, 6), vm.reshape(self.E, 8)

    def adjoint_dJdE(self, U, Lam, props=None):
        props = self.props if props is None else np.ascontiguousarray(props, dtype=np.float64)
        U = np.ascontiguousarray(np.atleast_2d(U), dtype=np.float64)
        Lam = np.ascontiguousarray(np.atleast_2d(Lam), dtype=np.float64)
        g = np.zeros(self.E)
        lib().orc_adjoint_dJdE(self.N, self.E, self.coords, self.conn, props, props.shape[1], U.shape[0], U, Lam, g)
        return g


def pcg(K: CSR, b, x0=None, rtol=1e-10, atol=0.0, max_iter=100000):
    x = np.zeros(K.n) if x0 is None else np.array(x0, dtype=np.float64)
    it = C.c_int(0)
    rf = C.c_double(0.0)
    ri = C.c_double(0.0)
    st = lib().orc_pcg(K.n, K.row_ptr, K.col, K.val, np.ascontiguousarray(b, dtype=np.float64), x, rtol, atol,
                       max_iter, C.byref(it), C.byref(rf), C.byref(ri))
    return x, {"status": st, "iters": it.value, "res_final": rf.value, "res_init": ri.value}


def pcg_marked(K: CSR, b, rtol=1e-13, mark_rtol=1e-10, max_iter=100000):
    """Jacobi-PCG from x0 = 0 to rtol, recording on the way the iterate, the
    iteration count and the wall time (setup included) at which the recursive
    residual first met mark_rtol: one run gives both the tightly converged
    reference solution and the time of the iter_pcg solve to mark_rtol
    (ufc_core/L2_NM/Solver/LinSolv/NM_Solv_IterSolver.f90:713-846)."""
    x = np.zeros(K.n)
    x_mark = np.zeros(K.n)
    it, it_mark = C.c_int(0), C.c_int(-1)
    rf, t_mark = C.c_double(0.0), C.c_double(-1.0)
    st = lib().orc_pcg_marked(K.n, K.row_ptr, K.col, K.val, np.ascontiguousarray(b, dtype=np.float64), x, rtol,
                              max_iter, mark_rtol, x_mark, C.byref(it_mark), C.byref(t_mark), C.byref(it),
                              C.byref(rf))
    return x, x_mark, {"status": st, "iters": it.value, "res_final": rf.value, "mark_iters": it_mark.value,
                       "mark_s": t_mark.value}


def nr_increment_j2(model: Model, u, state, tgt, tol=1e-8, max_iter=25, lin_rtol=1e-10):
    """One displacement-controlled J2 Newton-Raphson increment from the
    committed (u, state) to the prescribed values ``tgt``
    (RT_NLSolver_NewtonRaph, RT_Solv_Nonlin.f90:807-1002).  Each iteration
    updates every Gauss point from the committed state, assembles the
    consistent tangent and internal force, and solves K du = -R_free with
    Jacobi-PCG.  Convergence: ||R_free|| <= tol * max(||F_int||, 1e-30), F_int
    over every DOF (the reaction scale; the reference divides by ||F_ext||,
    RT_Step_NR_Core.f90:252-258, which is zero under displacement control),
    tested before each solve.  The first iteration of an increment is the
    predictor K_ff du_f = R_f - K_fc du_c (tangent at the start of the
    increment), after which the prescribed DOFs take their new values.
    Returns (converged, iterations, u, trial state, log); a non-finite residual
    or a failed linear solve is a non-convergence."""
    p = model.p
    u = u.copy()
    u_n = u.copy()
    free = np.ones(model.n, dtype=bool)
    free[p.fixed] = False
    dc = np.zeros(model.n)
    dc[p.fixed] = tgt - u[p.fixed]
    lift = bool(np.any(dc != 0.0))
    log = []
    trial = None
    for it in range(max_iter):
        fint, trial = model.fint_j2(u, u_n, state)
        R = -fint
        R[~free] = 0.0
        rn = np.linalg.norm(R)
        fn = max(np.linalg.norm(fint), 1e-30)
        log.append(rn / fn)
        if not np.isfinite(rn):
            return False, it, u, trial, log
        if not lift and rn <= tol * fn:
            return True, it, u, trial, log
        K = model.assemble(Dgp=trial["D"])
        if lift:
            y = model.assemble(Dgp=trial["D"], eliminate=False).matvec(dc)
            R[free] -= y[free]
        du, info = pcg(K, R, rtol=lin_rtol)
        if info["status"] != 0:
            return False, it, u, trial, log
        u += du
        if lift:
            u[p.fixed] = tgt
            lift = False
    return False, max_iter, u, trial, log


def nr_j2(model: Model, targets, tol=1e-8, max_iter=25, lin_rtol=1e-10):
    """Increments whose prescribed DOF values are ``targets`` (list of arrays),
    each solved by nr_increment_j2 from the previous converged one.  Returns
    the displacement history, the committed state and per-increment logs."""
    G = model.E * 8
    state = {"sig": np.zeros(G * 6), "epeq": np.zeros(G), "epl": np.zeros(G * 6)}
    u = np.zeros(model.n)
    hist, logs = [], []
    for tgt in targets:
        conv, _, u, trial, log = nr_increment_j2(model, u, state, tgt, tol, max_iter, lin_rtol)
        if not conv:
            raise RuntimeError("NR did not converge")
        state = {"sig": trial["sig"], "epeq": trial["epeq"], "epl": trial["epl"]}
        hist.append(u.copy())
        logs.append(log)
    return hist, state, logs


def step_j2(model: Model, u_end, time_period=1.0, dt_initial=1.0, dt_min=1e-5, dt_max=1.0, max_increments=100,
            max_cutbacks=5, auto_dt=True, target_iters=6, growth_threshold=0.8, growth_factor=1.25,
            cutback_factor=0.5, tol=1e-8, max_iter=25, lin_rtol=1e-10):
    """One step with automatic increments, from zero displacement and state to
    the prescribed values ``u_end`` ramped linearly in step time: the increment
    loop of RT_StepDriver_Execute (ufc_core/L5_RT/StepDriver/RT_Step_Exec.f90:415-600)
    with RT_StepDriver_End_Increment / RT_StepDriver_Cutback
    (RT_Step_Core.f90:215-300): after a converged increment dt grows by
    growth_factor when it took <= int(target_iters * growth_threshold) Newton
    iterations (capped by dt_max); a failed one is discarded and retried with
    dt * cutback_factor, the step failing below dt_min or after more than
    max_cutbacks consecutive cutbacks.  Returns a dict with the attempt history
    rows (time, dt, iterations, converged)."""
    p = model.p
    G = model.E * 8
    state = {"sig": np.zeros(G * 6), "epeq": np.zeros(G), "epl": np.zeros(G * 6)}
    u = np.zeros(model.n)
    u0 = u[p.fixed].copy()
    u_end = np.asarray(u_end, dtype=np.float64)
    T = float(time_period)
    t, dt = 0.0, min(dt_initial, dt_max)
    cut_run, attempts, increments, cutbacks, hist = 0, 0, 0, 0, []
    while t < T * (1.0 - 1e-12) and attempts < max_increments:
        dt = min(dt, T - t)
        t1 = t + dt
        s = 1.0 if t1 >= T else t1 / T
        tgt = u0 + s * (u_end - u0)
        conv, it, u_new, trial, _ = nr_increment_j2(model, u, state, tgt, tol, max_iter, lin_rtol)
        attempts += 1
        hist.append((t1, dt, it, conv))
        if conv:
            u = u_new
            state = {"sig": trial["sig"], "epeq": trial["epeq"], "epl": trial["epl"]}
            t = T if t1 >= T else t1
            increments += 1
            cut_run = 0
            if auto_dt and it <= int(target_iters * growth_threshold):
                dt = min(dt * growth_factor, dt_max)
            continue
        cutbacks += 1
        cut_run += 1
        if cut_run > max_cutbacks:
            break
        dt *= cutback_factor
        if dt < dt_min:
            break
    return {"completed": t >= T * (1.0 - 1e-12), "final_time": t, "history": hist, "u": u, "state": state,
            "increments": increments, "cutbacks": cutbacks, "attempts": attempts}
