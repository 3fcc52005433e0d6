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


def test_color_groups_follow_build_color_groups(pkg):
    """The colour groups of RT_AsmColor_Build (build_color_groups,
    RT_Asm_Color.f90:148-180), restated as its loops, against ufc_api's
    vectorised form on a random 1-based colouring."""
    import numpy as np

    color_of = np.random.default_rng(3).integers(1, 9, size=500).astype(np.int32)
    n = int(color_of.max())
    count = [0] * n
    for c in color_of:
        count[c - 1] += 1
    start = [1] * (n + 1)
    for c in range(n):
        start[c + 1] = start[c] + count[c]
    elems, fill = [0] * len(color_of), [0] * n
    for ie, c in enumerate(color_of, start=1):
        elems[start[c - 1] + fill[c - 1] - 1] = ie
        fill[c - 1] += 1
    got = pkg.ufc_api.color_groups(color_of)
    assert got[0] == n
    assert got[1].tolist() == count and got[2].tolist() == start and got[3].tolist() == elems
