"""Hand-written adjoint of the linear-elastic solve behind torch.autograd.

    U = UfcLinearElastic.apply(E, F, model, algo)

maps per-element Young's moduli E [n_elems] and nodal loads F ([n_dof] or
[nrhs, n_dof]) to displacements U of the same shape, solving K(E) U = P F on
the GPU with P the projection onto the free DOFs (Dirichlet values are zero).
Any scalar objective built from U and F by torch ops differentiates through it:
compliance J = sum(F * U), a tip displacement U[..., dof], ...

backward(gU) solves K Lam = P gU with the same PCG (Jacobi or multigrid
preconditioner, as algo says; K is symmetric),
reusing the stiffness assembled in forward and the saved U (nothing is
reassembled while E is unchanged), then evaluates
dJ/dE_e = -sum_k Lam_k,e^T (dK_e/dE_e) U_k,e for all elements in one kernel
(ufc_adjoint_sensitivity), and dJ/dF = P Lam.  The reference's adjoint is a
stub returning lambda = 0 (ufc_core/L2_NM/Solver/AI/NM_AI_AdjointAlgo.f90:116-136);
this follows the formulas of its contract K u = F, K^T lambda = dJ/du,
dJ/dtheta = -lambda^T dR/dtheta.  Density parametrisations (E = E0 rho^3) are
ordinary torch ops on top.
"""
from __future__ import annotations

import torch

from . import _abi as A
from .fem import FemModel, SolverAlgo

# largest block of right-hand sides ufc_pcg_solve_block takes in one call
MAX_BLOCK_RHS = 32


class ElasticModel:
    """A FemModel whose per-element moduli can change between solves."""

    def __init__(self, problem, device=0, build=A.BUILD_FP64):
        self.p = problem
        self.fem = FemModel.from_problem(problem, device=device)
        self.nu = torch.as_tensor(problem.props[:, 1], dtype=torch.float64)
        self.build = build
        self._E_key = None
        self.free = torch.ones(problem.n_dof, dtype=torch.float64)
        self.free[torch.as_tensor(problem.fixed, dtype=torch.long)] = 0.0
        self.free = self.free.to(torch.device("cuda", device))

    def set_moduli(self, E: torch.Tensor):
        """Reassemble K for new moduli; a no-op when E equals the moduli of the
        current assembly (compared by value: freed tensors reuse addresses)."""
        Ed = E.detach().to(torch.float64)
        if self._E_key is not None and self._E_key.shape == Ed.shape and torch.equal(self._E_key, Ed):
            return False
        props = torch.stack([Ed.cpu(), self.nu], dim=1).contiguous()
        self.fem.set_material(A.MAT_ELASTIC_ISO, props.numpy())
        self.fem.assemble(self.build)
        self._E_key = Ed.clone()
        return True

    def solve(self, B: torch.Tensor, algo: SolverAlgo):
        """Solve K X = P B for each row of B ([nrhs, n] or [n]).  With the
        Jacobi preconditioner, 2 to 32 right-hand sides are solved together by
        the block PCG (ufc_pcg_solve_block: one pass over K per iteration for
        all of them, each with its own recurrence and stop test); with the
        multigrid preconditioner, or more than 32, one after another."""
        single = B.dim() == 1
        B2 = (B.reshape(-1, B.shape[-1]) * self.free).contiguous()
        nrhs = B2.shape[0]
        if nrhs == 1:
            X, st = self.fem.solve(B2[0], algo)
            X, states = X.reshape(1, -1), [st]
        elif algo.precond_type == A.SOLV_PREC_JACOBI and nrhs <= MAX_BLOCK_RHS:
            X, states = self.fem.solve_block(B2, algo)
        else:
            X = torch.empty_like(B2)
            states = []
            for k in range(nrhs):
                _, st = self.fem.solve(B2[k], algo, x=X[k])
                states.append(st)
        self.last_states = states
        return (X[0] if single else X), states


class UfcLinearElastic(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, F, model: ElasticModel, algo: SolverAlgo | None = None):
        algo = algo or SolverAlgo(tolerance=1e-12)
        model.set_moduli(E)
        U, _ = model.solve(F.detach(), algo)
        ctx.model, ctx.algo = model, algo
        ctx.save_for_backward(E, U)
        return U

    @staticmethod
    def backward(ctx, gU):
        E, U = ctx.saved_tensors
        model, algo = ctx.model, ctx.algo
        model.set_moduli(E)  # no-op unless E changed since forward
        Lam, _ = model.solve(gU.contiguous(), algo)
        gE = gF = None
        if ctx.needs_input_grad[0]:
            U2 = U.reshape(-1, U.shape[-1]).contiguous()
            L2 = Lam.reshape(-1, Lam.shape[-1]).contiguous()
            gE = model.fem.adjoint_sensitivity(U2, L2).to(E.dtype)
        if ctx.needs_input_grad[1]:
            gF = Lam * model.free
        return gE, gF, None, None


def compliance(E, F, model, algo=None):
    """J = sum_k F_k . U_k with U = K(E)^-1 P F."""
    U = UfcLinearElastic.apply(E, F, model, algo)
    return (F * U).sum(), U


def density_objectives(rho, F, model, algo=None, tip_dof=None, E0=210e3, power=3.0):
    """The two objectives of a density problem, summed over its load cases
    (rows of F): compliance J1 = sum_k F_k . U_k and, when tip_dof is given,
    the displacement J2 = sum_k U_k[tip_dof], with U = K(E0 rho^power)^-1 P F
    solved by UfcLinearElastic (one block solve for up to 32 Jacobi cases).
    Returns (J1, J2 or None, U)."""
    U = UfcLinearElastic.apply(E0 * rho ** power, F, model, algo)
    J1 = (F * U).sum()
    J2 = U[..., tip_dof].sum() if tip_dof is not None else None
    return J1, J2, U


def central_differences(model, rho, F, U0, elems, algo, tip_dof=None, h=1e-6, E0=210e3, power=3.0):
    """Central finite differences of the density_objectives with respect to
    rho at the elements `elems` (a gradient check of the adjoint).  Each
    perturbed displacement is solved as a correction K' D = P (F - K' U0) from
    the unperturbed U0 ([nrhs, n]), and the two perturbed objectives are
    differenced through their corrections alone, so the difference is not
    swamped by the solver tolerance.  The moduli of rho are restored on exit.
    Returns (dJ1/drho, dJ2/drho) at the elements (the second None without
    tip_dof), as host lists."""
    F2 = F.reshape(-1, F.shape[-1])
    U2 = U0.reshape(-1, U0.shape[-1]).detach()
    base = rho.detach()
    d1, d2 = [], []
    try:
        for e in elems:
            vals = []
            for sgn in (1.0, -1.0):
                r = base.clone()
                r[int(e)] += sgn * h
                model.set_moduli(E0 * r ** power)
                R = torch.empty_like(U2)
                for k in range(U2.shape[0]):
                    _, R[k], _, _ = model.fem.internal_force(U2[k].contiguous(), f_ext=F2[k].contiguous(),
                                                             update_state=False)
                D, _ = model.solve(R, algo)
                vals.append(((F2 * D).sum().item(), D[:, tip_dof].sum().item() if tip_dof is not None else 0.0))
            d1.append((vals[0][0] - vals[1][0]) / (2 * h))
            d2.append((vals[0][1] - vals[1][1]) / (2 * h))
    finally:
        model.set_moduli(E0 * base ** power)
    return d1, (d2 if tip_dof is not None else None)
