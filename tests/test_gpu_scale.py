"""Full-size checks on the 128x64x64 and 192x96x96 lognormal cantilevers, the
adjoint at 128x64x64 and the J2 bar at 64x32x32, through properties that do not
need the oracle at that size: an independent FP64 residual (matrix-free element
operator against the assembled-matrix solve), agreement of the FP32+refine,
FP64 and symmetric-storage solutions, the compliance identity f.u = u.K.u,
bitwise reproducibility, and adjoint gradients against finite differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(pkg):
    import torch

    out = {}
    for name, make in (("128x64x64", pkg.mesh.config2), ("192x96x96", pkg.mesh.config4)):
        p = make()
        m = pkg.FemModel.from_problem(p)
        m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
        b = torch.from_numpy(pkg.lifted_rhs(m, p.f)).cuda()
        out[name] = (p, m, b)
    yield out
    for _, m, _ in out.values():
        m.close()


@pytest.mark.parametrize("name", ["128x64x64", "192x96x96"])
def test_full_size_fp64_and_mixed(pkg, big, name):
    import torch

    p, m, b = big[name]
    u64, s64 = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    u32, s32 = m.solve(b, pkg.SolverAlgo(tolerance=1e-10, precision_mode=pkg.PRECISION_FP32_REFINE))
    assert s64.converged and s32.converged and s64.rnorm <= 1e-10 and s32.rnorm <= 1e-10
    bn = torch.linalg.vector_norm(b).item()
    for u in (u64, u32):
        # independent residual: matrix-free FP64 element operator, not the assembled matrix
        _, r, rn, _ = m.internal_force(u, f_ext=b)
        assert rn / bn <= 1.5e-10
    rel = (torch.linalg.vector_norm(u32 - u64) / torch.linalg.vector_norm(u64)).item()
    assert rel <= 1e-9, rel
    # compliance identity f.u = u.K.u (energy), through the SpMV
    Ku = m.spmv(u64)
    assert abs(torch.dot(b, u64).item() - torch.dot(u64, Ku).item()) <= 1e-9 * abs(torch.dot(b, u64).item())
    # von Mises of the two solutions
    _, vm64 = m.stress(u64, want_sigma=False)
    _, vm32 = m.stress(u32, want_sigma=False)
    assert (torch.max(torch.abs(vm32 - vm64)) / torch.max(vm64)).item() <= 1e-8
    # bitwise reproducible solve
    u64b, _ = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    assert torch.equal(u64, u64b)


def test_symmetric_storage_full_size(pkg, big):
    import torch

    p, m, b = big["128x64x64"]
    u_full, _ = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED | pkg.BUILD_SYMMETRIC)
    try:
        u_sym, s = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
        assert s.converged
        assert (torch.linalg.vector_norm(u_sym - u_full) / torch.linalg.vector_norm(u_full)).item() <= 1e-9
        x = torch.randn(p.n_dof, dtype=torch.float64, device="cuda")
        y_sym = m.spmv(x)
    finally:
        m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
    y_full = m.spmv(x)
    assert (torch.max(torch.abs(y_sym - y_full)) / torch.max(torch.abs(y_full))).item() <= 1e-13


def test_adjoint_block_128x64x64(pkg):
    """16 tip-load cases solved as one block; compliance gradients dJ/drho of the
    first case against central finite differences (h = 1e-6) on 4 of the 32
    seeded elements, each finite difference solved as a correction."""
    import torch

    from ufc_fem_kernel_b200.adjoint import ElasticModel

    p = pkg.mesh.config5()
    dev = torch.device("cuda", 0)
    model = ElasticModel(p, device=0)
    rho = torch.tensor(p.meta["rho"], dtype=torch.float64, device=dev)
    F = torch.tensor(p.meta["F"], dtype=torch.float64, device=dev)
    model.set_moduli(210e3 * rho ** 3)
    algo = pkg.SolverAlgo(tolerance=1e-10)
    U, states = model.fem.solve_block(F * model.free, algo)
    assert all(s.converged for s in states) and len(states) == 16
    u0, s0 = model.fem.solve(F[0] * model.free, algo)
    assert (torch.linalg.vector_norm(U[0] - u0) / torch.linalg.vector_norm(u0)).item() <= 1e-8
    # compliance of case 0: lambda = u, dJ/dE_e = -u_e^T (K_e/E_e) u_e, chain rule to rho
    gE = model.fem.adjoint_sensitivity(U[:1].contiguous(), U[:1].contiguous())
    g = gE * 3 * 210e3 * rho ** 2
    h = 1e-6
    for e in p.meta["fd_elems"][:4]:
        d = []
        for sgn in (1.0, -1.0):
            rp = rho.clone()
            rp[e] += sgn * h
            model.set_moduli(210e3 * rp ** 3)
            _, r, _, _ = model.fem.internal_force(U[0].contiguous(), f_ext=(F[0] * model.free).contiguous(),
                                                  update_state=False)
            du, _ = model.fem.solve(r, pkg.SolverAlgo(tolerance=1e-10))
            d.append(torch.dot(F[0], du).item())
        fd = (d[0] - d[1]) / (2 * h)
        assert abs(g[e].item() - fd) <= 1e-6 * abs(fd), (int(e), g[e].item(), fd)
    model.set_moduli(210e3 * rho ** 3)
