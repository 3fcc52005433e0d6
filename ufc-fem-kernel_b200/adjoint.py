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
        """Solve K X = P B for each row of B ([nrhs, n] or [n])."""
        single = B.dim() == 1
        B2 = (B.reshape(-1, B.shape[-1]) * self.free).contiguous()
        if B2.shape[0] == 1:
            X, st = self.fem.solve(B2[0], algo)
            X, states = X.reshape(1, -1), [st]
        else:
            X = torch.empty_like(B2)
            states = []
            for k in range(B2.shape[0]):
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
