"""Host side of the reference call surface (ufc_api), on the CPU: the bundles'
defaults and the argument checks of NM_Solver_Algo_SetTol / SetMaxIter
(ufc_core/L2_NM/Solver/NM_Solv_Def.f90:187-207)."""
import pytest


def test_bundles_and_setters(pkg):
    api = pkg.ufc_api
    algo = api.NM_Solver_Algo()
    assert algo.method == api.NM_SOLV_METHOD_CG and algo.precond_type == api.NM_SOLV_PREC_JACOBI
    algo.SetTolerance(1e-9)
    algo.SetMaxIter(50)
    assert algo.tolerance == 1e-9 and algo.max_iter == 50
    with pytest.raises(ValueError, match="Tolerance must be positive"):
        algo.SetTolerance(0.0)
    with pytest.raises(ValueError, match="Max iterations must be >= 1"):
        algo.SetMaxIter(0)
    # the algo converts to the C struct the library reads
    c = algo.to_c()
    assert c.max_iter == 50 and c.tolerance == 1e-9
    st = api.init_error_status(api.ErrorStatusType(4, "x", "y"))
    assert st.ok and st.message == "" and st.source == ""
    assert api.NM_Solver_State().residual_history is None and not api.NM_Solver_State().converged
    assert api.MD_NonlinSolv().tolerance_force == 1e-8 and api.MD_NonlinSolv().max_iterations == 25


def test_pcg_rejects_missing_rhs_without_a_device(pkg):
    """Argument errors are statuses, found before anything runs."""
    api = pkg.ufc_api

    class NoModel:
        n_dof = 9

    status = api.NM_Solver_PCG(api.NM_Solver_Desc(n=9), api.NM_Solver_State(), api.NM_Solver_Algo(),
                               api.NM_Solver_Ctx(NoModel()))
    assert status.status_code == api.IF_STATUS_INVALID and "state%b" in status.message
    status = api.NM_Solver_PCG(api.NM_Solver_Desc(n=10), api.NM_Solver_State(b=[0.0] * 9), api.NM_Solver_Algo(),
                               api.NM_Solver_Ctx(NoModel()))
    assert status.status_code == api.IF_STATUS_INVALID and "desc%n" in status.message
