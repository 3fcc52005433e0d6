"""Time-to-rtol 1e-10 of Jacobi-PCG on the 192x96x96 C3D8 cantilever (5,447,811 DOF).

One step = one linear static solve K u = f on one GPU, from x0 = 0 to
||f - K u||_2 <= 1e-10 ||f||_2 in FP64, with the stiffness already assembled in
HBM (pattern and assembly are timed separately and reported in `assembly`).
The headline (`value`) is the FP32 matrix / FP64-refined PCG; the plain FP64
PCG on the same mesh is timed in the same run (`fp64_path`).  Both use the
symmetric half storage of the block matrix by default (`--storage full` for
the full SELL-32 storage, which is also timed once as `other_storage`).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun, one rank per GPU): every rank solves its own copy of the
problem (replicas; the path is a single-GPU solve), the reported time is the
maximum over ranks.

`--impl reference` times the CPU FP64 Jacobi-PCG of the oracle (the
restatement of the reference's Fortran iter_pcg, which has no buildable form
here) on the host cores: whole solves of the same problem from x0 = 0 to rtol
1e-10, timed in full.  The `cpu_baseline` of the GPU line is the same solve,
measured on the way of one oracle run continued to rtol 1e-13, whose solution
is the reference for `accuracy_vs_oracle` (displacement and von Mises errors of
every GPU solution).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-rtol 1e-10, 5.4M-DOF C3D8: FP32+FP64-refine vs FP64 PCG, 1 B200"
UNIT = "s"
WORKLOAD = ("C3D8 cantilever 192x96x96 unit hexes (1,769,472 elements, 5,447,811 DOF, 433,724,553 nnz), "
            "lognormal E (mu ln 210e3, sigma 0.5, seed 4), nu 0.3, clamped x=0, traction (0,0,-1) on x=192; "
            "Jacobi-PCG from x0=0 to ||f-Ku||/||f|| <= 1e-10 (FP64 residual)")


def workload(mesh):
    """The workload text of a --mesh other than the 192x96x96 default."""
    if mesh == "192x96x96":
        return WORKLOAD
    nx, ny, nz = mesh_dims(mesh)
    n_dof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    return (f"C3D8 cantilever {mesh} unit hexes ({nx * ny * nz:,} elements, {n_dof:,} DOF), lognormal E "
            f"(mu ln 210e3, sigma 0.5, seed 4), nu 0.3, clamped x=0, traction (0,0,-1) on x={nx}; Jacobi-PCG from "
            "x0=0 to ||f-Ku||/||f|| <= 1e-10 (FP64 residual)")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mesh", default="192x96x96", help="nx x ny x nz of the lognormal cantilever")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the J2 bar and adjoint block workloads reported under `other_configs`")
    ap.add_argument("--cpu-iters", type=int, default=12, help="CG iterations per warm-up sample of the CPU arm")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="seconds of whole CPU solves the reference arm times after the first one")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--storage", choices=["symmetric", "full"], default="symmetric",
                    help="block storage of both paths: symmetric half (default) or full SELL-32")
    return ap.parse_args(argv)


def _dist_active():
    try:
        import torch.distributed as td

        return td.is_available() and td.is_initialized() and td.get_world_size() > 1
    except Exception:
        return False


def barrier(device=None):
    """Process-group barrier (when one is initialised), then a device synchronize."""
    import torch

    if _dist_active():
        import torch.distributed as td

        td.barrier()
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)


def max_over_ranks(value, device=None):
    """Maximum of a per-rank float over the process group (identity on one rank).
    The tensor lives on `device` (a CUDA device under NCCL, the CPU under gloo)."""
    if not _dist_active():
        return float(value)
    import torch
    import torch.distributed as td

    t = torch.tensor([float(value)], dtype=torch.float64, device=device if device is not None else "cpu")
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(name):
    """DRAM bytes per launch recorded in profiles/<name> (a 'traffic_bytes_per_launch:' line)."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(float(line.split(":", 1)[1].split()[0]))
    except Exception:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="ufc_clocks_", suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def mesh_dims(s):
    return tuple(int(v) for v in s.lower().split("x"))


def make_problem(args):
    import __graft_entry__ as g

    ufc = g.load_package()
    nx, ny, nz = mesh_dims(args.mesh)
    return ufc, ufc.mesh.lognormal_cantilever(nx, ny, nz, seed=4)


def oracle_reference(p, solutions=None, vm=None, gpu_csr=None, rtol=1e-13, mark_rtol=1e-10, props=None):
    """The oracle's own FP64 Jacobi-PCG solve of the problem on all host
    threads, from x0 = 0, continued to the recursive rtol `rtol` for a
    reference solution; the wall time and iterate at which it first met
    `mark_rtol` are those of the iter_pcg solve to mark_rtol (the CPU
    baseline, measured in full).  Each GPU solution in `solutions` (name ->
    host array) is compared with the reference solution: relative L2 and max
    displacement error, ||b - K u|| / ||b|| with the oracle's CSR and lifted
    b, and, when `vm` holds that solution's Gauss-point von Mises stress from
    the GPU ([E, 8]), the largest von Mises difference relative to the largest
    reference value.  gpu_csr, when given, returns the GPU's exported
    canonical CSR (row_ptr, col, FP64 values), compared with the oracle's:
    pattern equality and the largest value difference relative to the largest
    entry.  Returns (cpu_baseline, accuracy)."""
    from oracle import oracle as O

    import numpy as np

    t0 = time.perf_counter()
    model = O.Model(p)
    K = model.assemble(props=props)
    b = model.lifted_rhs()
    setup = time.perf_counter() - t0
    acc = {}
    if gpu_csr is not None:
        rp, col, v = gpu_csr()
        same = bool(np.array_equal(rp, K.row_ptr) and np.array_equal(col, K.col))
        acc["csr"] = {"pattern_equal": same, "nnz": int(col.size),
                      "values_rel_max_err": float(np.abs(v - K.val).max() / np.abs(K.val).max()) if same else None}
        del rp, col, v
    t = time.perf_counter()
    u_ref, u_mark, info = O.pcg_marked(K, b, rtol=rtol, mark_rtol=mark_rtol)
    total = time.perf_counter() - t
    bn = float(np.linalg.norm(b))
    un = float(np.linalg.norm(u_ref))
    umax = float(np.abs(u_ref).max())
    vm_ref = model.elastic_vm(u_ref, props=props)[1] if vm else None
    vmax = float(np.abs(vm_ref).max()) if vm_ref is not None else None

    def errors(u, vm_u=None):
        e = {"u_rel_l2": float(np.linalg.norm(u - u_ref) / un), "u_rel_max": float(np.abs(u - u_ref).max() / umax),
             "residual_rel": float(np.linalg.norm(b - K.matvec(u)) / bn)}
        if vm_u is not None and vm_ref is not None:
            e["von_mises_rel_max"] = float(np.abs(np.asarray(vm_u).reshape(vm_ref.shape) - vm_ref).max() / vmax)
        return e

    acc["reference"] = {
        "solver": f"oracle FP64 Jacobi-PCG (iter_pcg restated, canonical CSR, lifted b) from x0 = 0 to recursive "
                  f"rtol {rtol:g}", "iters": info["iters"], "true_residual_rel": errors(u_ref)["residual_rel"]}
    for name, u in (solutions or {}).items():
        acc[name] = errors(u, (vm or {}).get(name))
    acc[f"oracle_rtol_{mark_rtol:g}"] = errors(u_mark)
    cpu = {"value": info["mark_s"], "unit": UNIT, "cores": O.num_threads(), "kind": "port",
           "sample": f"the whole FP64 Jacobi-PCG solve of the oracle (OpenMP, canonical CSR) from x0 = 0 to rtol "
                     f"{mark_rtol:g}: {info['mark_iters']} iterations, measured on the way of one run continued to "
                     f"{rtol:g} ({info['iters']} iterations, {total:.1f} s) for the reference solution; CPU CSR "
                     f"build {setup:.1f} s excluded"}
    return cpu, acc


def cpu_pcg_full(p, props=None, rtol=1e-10):
    """One whole FP64 Jacobi-PCG solve of the oracle from x0 = 0 to rtol on all
    host threads, timed (CSR build excluded): (seconds, iterations, threads)."""
    from oracle import oracle as O

    model = O.Model(p)
    K = model.assemble(props=props)
    b = model.lifted_rhs()
    t = time.perf_counter()
    _, info = O.pcg(K, b, rtol=rtol)
    return time.perf_counter() - t, info["iters"], O.num_threads()


def linear_static(ufc, local, p, cpu=False):
    """Time-to-rtol 1e-10 of one linear-elastic problem from x0 = 0: FP64
    Jacobi-PCG, the FP32+FP64-refined one (symmetric storage) and FP64 PCG with the
    multigrid preconditioner, each timed by the library's CUDA events after one
    warm-up solve, with the assembly time.  With cpu, the oracle solves the
    same problem on the host (the measured CPU baseline) to a tight tolerance,
    and each GPU solution's displacement and von Mises errors against it are
    reported under accuracy_vs_oracle."""
    import torch

    dev = torch.device("cuda", local)
    m = ufc.FemModel.from_problem(p, device=local)
    # the symmetric half storage, as the headline (coded indices where the mesh
    # has enough slices for the one-warp-per-slice product)
    ka = m.assemble(ufc.BUILD_FP64 | ufc.BUILD_FP32_ROUNDED | ufc.BUILD_SYMMETRIC)
    b = torch.from_numpy(ufc.lifted_rhs(m, p.f)).to(dev)
    x = torch.zeros_like(b)
    res = {"n_dof": p.n_dof, "elements": p.n_elems, "assembly_ms": ka}
    sols, vms = {}, {}
    for key, pm in (("fp64", ufc.PRECISION_FP64), ("fp32_refine", ufc.PRECISION_FP32_REFINE)):
        a = ufc.SolverAlgo(tolerance=1e-10, precision_mode=pm)
        x.zero_()
        m.solve(b, a, x=x, raise_on_not_converged=False)
        x.zero_()
        _, st = m.solve(b, a, x=x, raise_on_not_converged=False)
        res[key] = {"s": st.solve_time / 1e3, "iters": st.niter, "rnorm": st.rnorm, "converged": st.converged}
        if pm != ufc.PRECISION_FP64:
            res[key]["fp64_continuation_iters"] = st.fp64_iters
        if cpu:
            sols[key] = x.cpu().numpy()
            vms[key] = m.stress(x, want_sigma=False)[1].cpu().numpy()
    if res["fp32_refine"]["fp64_continuation_iters"] == res["fp32_refine"]["iters"]:
        # the matrix fits in L2, so the refined request ran FP64 iterations; the
        # FP32 iterations forced on the same problem, for comparison
        a = ufc.SolverAlgo(tolerance=1e-10, precision_mode=ufc.PRECISION_FP32_REFINE,
                           refine_policy=ufc.REFINE_FORCE_FP32)
        x.zero_()
        m.solve(b, a, x=x, raise_on_not_converged=False)
        x.zero_()
        _, st = m.solve(b, a, x=x, raise_on_not_converged=False)
        res["fp32_forced"] = {"s": st.solve_time / 1e3, "iters": st.niter, "rnorm": st.rnorm,
                              "converged": st.converged, "fp64_continuation_iters": st.fp64_iters,
                              "note": "FP32 iterations forced (UFC_REFINE_FORCE_FP32); fp32_refine ran FP64 "
                                      "iterations because the FP64 matrix is read from L2"}
    # FP64 PCG with the geometric multigrid V-cycle in FP32 (set-up outside the timed solve)
    levels, coarse, setup_ms = m.mg_setup(*p.shape, precision=ufc.PRECISION_FP32_REFINE)
    a = ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG)
    x.zero_()
    m.solve(b, a, x=x, raise_on_not_converged=False)
    x.zero_()
    _, st = m.solve(b, a, x=x, raise_on_not_converged=False)
    res["multigrid"] = {"s": st.solve_time / 1e3, "iters": st.niter, "rnorm": st.rnorm, "converged": st.converged,
                        "levels": levels, "coarsest_dof": coarse, "setup_s": setup_ms / 1e3}
    if cpu:
        sols["multigrid"] = x.cpu().numpy()
        vms["multigrid"] = m.stress(x, want_sigma=False)[1].cpu().numpy()
    m.close()
    if cpu:
        res["cpu_baseline"], res["accuracy_vs_oracle"] = oracle_reference(p, sols, vms)
    return res


def cpu_j2(p, nr_iters, cg_iters, sample_iters=12):
    """The oracle's cost of the J2 bar on the CPU (all host threads), from the
    parts of one Newton iteration: the return map and internal force at every
    Gauss point, the tangent assembly, and sample_iters FP64 Jacobi-PCG
    iterations on that tangent, extrapolated to the GPU run's Newton and CG
    iteration counts."""
    import numpy as np

    from oracle import oracle as O

    model = O.Model(p)
    G = model.E * 8
    state = {"sig": np.zeros(G * 6), "epeq": np.zeros(G), "epl": np.zeros(G * 6)}
    u = np.zeros(model.n)
    t = time.perf_counter()
    _, trial = model.fint_j2(u, u, state)
    K = model.assemble(Dgp=trial["D"])
    t_nr = time.perf_counter() - t
    b = np.random.default_rng(0).standard_normal(model.n)  # any right-hand side: only the time is used
    b[p.fixed] = 0.0
    t = time.perf_counter()
    O.pcg(K, b, max_iter=-sample_iters)
    per = (time.perf_counter() - t) / sample_iters
    return {"s": nr_iters * t_nr + cg_iters * per, "kind": "port", "cores": O.num_threads(),
            "sample": f"one return map + tangent assembly ({t_nr:.3f} s) x {nr_iters} Newton iterations + "
                      f"{sample_iters} PCG iterations ({per * 1e3:.2f} ms/iter) x {cg_iters}"}


def cpu_adjoint(p, E, F, U):
    """The oracle's cost of the 16-case adjoint workload on the CPU (all host
    threads): load case 0 solved in full by FP64 Jacobi-PCG from x0 = 0 to rtol
    1e-10 (measured) times the number of cases, plus the sensitivity dJ/dE of
    all cases, timed in full."""
    import numpy as np

    from oracle import oracle as O

    model = O.Model(p)
    props = np.stack([E, p.props[:, 1]], axis=1)
    K = model.assemble(props=props)
    b = np.ascontiguousarray(F[0])
    t = time.perf_counter()
    _, info = O.pcg(K, b, rtol=1e-10)
    t_case = time.perf_counter() - t
    t = time.perf_counter()
    model.adjoint_dJdE(U, U, props=props)
    t_sens = time.perf_counter() - t
    n = U.shape[0]
    return {"s": n * t_case + t_sens, "kind": "port", "cores": O.num_threads(),
            "sample": f"load case 0 solved in full ({info['iters']} iterations, {t_case:.1f} s, measured) x {n} "
                      f"cases + the sensitivity of all {n} cases ({t_sens:.3f} s, measured)"}


def adjoint_workload(ufc, local, stream, cpu=False):
    """The 128x64x64 density problem (E = 210e3 rho^3) with 16 tip-load cases
    through UfcLinearElastic (torch.autograd): the forward solve of all 16
    cases, then dJ/drho and dJ/dF of both objectives summed over the cases,
    compliance J1 = sum f.u and the tip-centre displacement J2 = sum u_z(tip),
    each backward one adjoint solve of the 16 cases plus the sensitivity
    kernel.  Timed with CUDA events once with the Jacobi block PCG (all 16
    cases per SpMV pass) and once with the multigrid PCG (cases one after
    another).  Checked against central differences (h = 1e-6) on the 32
    seeded elements for both objectives, and dJ2/dF by linearity."""
    import torch

    from ufc_fem_kernel_b200.adjoint import ElasticModel, central_differences, density_objectives

    dev = torch.device("cuda", local)
    p = ufc.mesh.config5()
    model = ElasticModel(p, device=local)
    rho0 = torch.tensor(p.meta["rho"], dtype=torch.float64, device=dev)
    F0 = torch.tensor(p.meta["F"], dtype=torch.float64, device=dev) * model.free
    tip = 3 * int(p.meta["tip_node"]) + 2
    model.set_moduli(210e3 * rho0 ** 3)
    model.fem.mg_setup(*p.shape, precision=ufc.PRECISION_FP32_REFINE)
    algos = {"jacobi_block": ufc.SolverAlgo(tolerance=1e-10),
             "multigrid": ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG)}
    res = {"workload": "density problem 128x64x64 (E = 210e3 rho^3, rho ~ U(0.3,1), seed 5), 16 tip-load cases; "
                       "UfcLinearElastic forward (K U = P F, rtol 1e-10) and torch.autograd backward of J1 = sum f.u "
                       "(compliance) and J2 = sum u_z(tip-centre node): dJ/drho (524,288 values) and dJ/dF",
           "n_dof": p.n_dof}
    grads = {}
    for name, algo in algos.items():
        ts = None
        for rep in range(2):  # the first pass warms up (graphs, multigrid refresh)
            rho = rho0.clone().requires_grad_(True)
            F = F0.clone().requires_grad_(True)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            torch.cuda.synchronize(dev)
            ev[0].record(stream)
            J1, J2, U = density_objectives(rho, F, model, algo, tip)
            ev[1].record(stream)
            g1 = torch.autograd.grad(J1, [rho, F], retain_graph=True)
            ev[2].record(stream)
            g2 = torch.autograd.grad(J2, [rho, F])
            ev[3].record(stream)
            torch.cuda.synchronize(dev)
            ts = [ev[k].elapsed_time(ev[k + 1]) / 1e3 for k in range(3)]
        st = model.last_states
        res[name] = {"forward_s": ts[0], "backward_J1_s": ts[1], "backward_J2_s": ts[2], "total_s": sum(ts),
                     "iters_max_last_solve": max(s.niter for s in st),
                     "converged": all(s.converged for s in st)}
        grads[name] = (g1[0].detach(), g2[0].detach(), g2[1].detach(), U.detach(), J2.item())
    gj, gm = grads["jacobi_block"], grads["multigrid"]
    res["multigrid_vs_block"] = {
        "u_rel": (torch.linalg.vector_norm(gm[3] - gj[3]) / torch.linalg.vector_norm(gj[3])).item(),
        "dJ1_drho_rel": (torch.linalg.vector_norm(gm[0] - gj[0]) / torch.linalg.vector_norm(gj[0])).item(),
        "dJ2_drho_rel": (torch.linalg.vector_norm(gm[1] - gj[1]) / torch.linalg.vector_norm(gj[1])).item()}
    # central differences on the 32 seeded elements, both objectives (multigrid corrections)
    elems = [int(e) for e in p.meta["fd_elems"]]
    fd1, fd2 = central_differences(model, rho0, F0, gj[3], elems, algos["multigrid"], tip_dof=tip)
    e1 = max(abs(gj[0][e].item() - f) / abs(f) for e, f in zip(elems, fd1))
    scale2 = gj[1].abs().max().item()
    e2 = max(abs(gj[1][e].item() - f) / max(abs(f), 1e-12 * scale2) for e, f in zip(elems, fd2))
    # dJ2/dF by linearity: J2(F + d) - J2(F) = d . dJ2/dF exactly
    d = torch.randn(F0.shape, generator=torch.Generator(device=dev).manual_seed(7), device=dev,
                    dtype=torch.float64) * model.free
    with torch.no_grad():
        _, J2d, _ = density_objectives(rho0, F0 + d, model, algos["jacobi_block"], tip)
    lin = abs((J2d.item() - gj[4]) - torch.sum(d * gj[2]).item()) / abs(torch.sum(d * gj[2]).item())
    res["fd_check"] = {"elements": len(elems), "h": 1e-6, "max_rel_err_J1": e1, "max_rel_err_J2": e2,
                       "dJ2_dF_linearity_rel_err": lin,
                       "note": "autograd dJ/drho (Jacobi block PCG) against central differences, each perturbed "
                               "solve a multigrid correction from the unperturbed U"}
    if cpu:
        res["cpu_baseline"] = cpu_adjoint(p, 210e3 * rho0.cpu().numpy() ** 3, F0.cpu().numpy(),
                                          gj[3].cpu().numpy())
    model.fem.close()
    return res


def other_configs(ufc, local, stream, cpu=False):
    """The other device workloads of the path, timed with CUDA events: the
    40x8x8 cantilever and the 128x64x64 lognormal cantilever (linear static),
    the 64x32x32 J2 bar pulled to 1 % strain in 20 Newton-Raphson increments, and
    16 tip-load cases of the 128x64x64 density problem solved as one block PCG
    plus the adjoint sensitivity dJ/dE of every element."""
    import torch

    dev = torch.device("cuda", local)
    out = {}
    for key, make in (("cantilever_40x8x8", ufc.mesh.config1), ("lognormal_128x64x64", ufc.mesh.config2)):
        try:
            out[key] = linear_static(ufc, local, make(), cpu)
        except Exception as e:  # a failure here must not lose the headline line
            out[key] = {"error": f"{type(e).__name__}: {e}"}
    try:
        p = ufc.mesh.config3()

        def j2_run(multigrid, n_steps):
            """The first n_steps of the 20 increments on a fresh model, timed with
            CUDA events: (seconds, converged, Newton iterations, CG iterations)."""
            m = ufc.FemModel.from_problem(p, device=local)
            lin = ufc.SolverAlgo(tolerance=1e-10)
            if multigrid:  # hierarchy built once, its numbers rebuilt after every tangent assembly
                m.internal_force(m.displacement(), update_state=True)
                m.assemble(ufc.BUILD_FP64)
                m.mg_setup(*p.shape)
                lin = ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            torch.cuda.synchronize(dev)
            ev[0].record(stream)
            nr_iters = lin_iters = 0
            ok = True
            for s in range(1, n_steps + 1):
                res = m.nr_increment(ufc.mesh.j2_bar_target(p, s), tolerance_force=1e-8, lin=lin)
                ok = ok and res.converged
                nr_iters += res.iterations
                lin_iters += res.lin_iters_total
                m.commit()
            ev[1].record(stream)
            torch.cuda.synchronize(dev)
            m.close()
            return ev[0].elapsed_time(ev[1]) / 1e3, ok, nr_iters, lin_iters

        # warm-up: the first elastic and plastic increments of each variant on a
        # throwaway model (first kernel launches, graph paths), then the timed run
        for mg in (False, True):
            j2_run(mg, 5)
        t, ok, nr_iters, lin_iters = j2_run(False, 20)
        out["j2_bar_64x32x32"] = {
            "workload": "J2 bar 64x32x32 (E 200e3, nu 0.3, sy 250, H 1000), 20 displacement increments to 1 % "
                        "strain, NR to ||r|| <= 1e-8 max(||F_ext||,||F_int||), FP64 PCG rtol 1e-10 per iteration",
            "s": t, "converged": ok, "nr_iterations": nr_iters,
            "pcg_iterations": lin_iters, "n_dof": p.n_dof, "preconditioner": "Jacobi"}
        t, ok, nr_iters, lin_iters = j2_run(True, 20)
        out["j2_bar_64x32x32_multigrid"] = {
            "s": t, "converged": ok, "nr_iterations": nr_iters,
            "pcg_iterations": lin_iters, "preconditioner": "geometric multigrid (FP64 V-cycle), numerics rebuilt "
                                                          "after every tangent assembly"}
        if cpu:
            out["j2_bar_64x32x32"]["cpu_baseline"] = cpu_j2(p, out["j2_bar_64x32x32"]["nr_iterations"],
                                                           out["j2_bar_64x32x32"]["pcg_iterations"])
    except Exception as e:  # a failure here must not lose the headline line
        out["j2_bar_64x32x32"] = {"error": f"{type(e).__name__}: {e}"}
    try:
        out["adjoint_128x64x64_16rhs"] = adjoint_workload(ufc, local, stream, cpu)
    except Exception as e:
        out["adjoint_128x64x64_16rhs"] = {"error": f"{type(e).__name__}: {e}"}
    return out


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    """The CPU arm: the oracle's FP64 Jacobi-PCG (the reference's iter_pcg
    restated; the Fortran cannot be built here) on all host threads.  Warm-up
    steps are short samples of --cpu-iters iterations; each timed step is one
    whole solve from x0 = 0 to rtol 1e-10, and as many whole solves are timed
    as fit in --ref-budget seconds (at least one), so the reported time is
    measured, not extrapolated.  Rank 0 alone works under torchrun."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    _, p = make_problem(args)
    t0 = time.perf_counter()
    model = O.Model(p)
    K = model.assemble()
    b = model.lifted_rhs()
    setup = time.perf_counter() - t0
    threads = O.num_threads()
    for _ in range(args.warmup):
        O.pcg(K, b, max_iter=-args.cpu_iters)
    times, iters = [], []
    t_begin = time.perf_counter()
    while True:
        t = time.perf_counter()
        _, info = O.pcg(K, b, rtol=1e-10)
        times.append(time.perf_counter() - t)
        iters.append(info["iters"])
        spent = time.perf_counter() - t_begin
        if len(times) >= args.steps or spent + times[-1] > args.ref_budget:
            break
    value = statistics.median(times)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, numpy)",
            "config": {"workload": workload(args.mesh), "parallelism": "host threads", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{len(times)} whole FP64 Jacobi-PCG solve(s) of the oracle (OpenMP, canonical "
                                       f"CSR) from x0 = 0 to rtol 1e-10, {iters[-1]} iterations each, timed in full "
                                       f"(median); warm-up: {args.warmup} samples of {args.cpu_iters} iterations; CSR "
                                       f"build {setup:.1f} s excluded"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    world, rank, local = dist_env()
    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as td

        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    ufc, p = make_problem(args)
    t0 = time.perf_counter()
    m = ufc.FemModel.from_problem(p, device=local, build_pattern=False)
    setup_s = time.perf_counter() - t0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    info = m.pattern_build()
    ev[1].record(stream)
    torch.cuda.synchronize(dev)
    pattern_ms = ev[0].elapsed_time(ev[1])
    sym = args.storage == "symmetric"
    build = ufc.BUILD_FP64 | ufc.BUILD_FP32_ROUNDED | (ufc.BUILD_SYMMETRIC if sym else 0)
    asm_ms = m.assemble(ufc.BUILD_FP64 | ufc.BUILD_FP32_ROUNDED)
    asm32_ms = m.assemble(ufc.BUILD_FP32)  # FP32 element kernel, timed for the elements/s figure
    asm_ms = m.assemble(ufc.BUILD_FP64 | ufc.BUILD_FP32_ROUNDED)
    build_ms = m.assemble(build)

    b_host = ufc.lifted_rhs(m, p.f)
    b = torch.from_numpy(b_host).to(dev)
    x = torch.zeros_like(b)
    mixed = ufc.SolverAlgo(tolerance=1e-10, precision_mode=ufc.PRECISION_FP32_REFINE, refine_delta=0.1)
    fp64 = ufc.SolverAlgo(tolerance=1e-10, precision_mode=ufc.PRECISION_FP64)

    # ---- warm-up, then the timed steps (device-resident inputs)
    for _ in range(args.warmup):
        m.solve(b, mixed, x=x)
    clocks = Clocks(local)
    barrier(dev)
    clocks.start()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    states = []
    launches = 0
    evs[0].record(stream)
    for k in range(args.steps):
        _, st = m.solve(b, mixed, x=x)
        evs[k + 1].record(stream)
        states.append(st)
        launches += m.last_timing()["kernel_launches"]
    barrier(dev)
    clk = clocks.stop()
    step_s = [evs[k].elapsed_time(evs[k + 1]) / 1e3 for k in range(args.steps)]
    t_mixed = max_over_ranks(sum(step_s) / len(step_s), dev)
    u_mixed = x.clone()

    # ---- SpMV roofline: instrumented solve (CUDA events around every SpMV launch)
    m.set_instrument(True)
    m.solve(b, mixed, x=x)
    tm = m.last_timing()
    m.set_instrument(False)
    spmv_avg_s = tm["spmv_ms"] / tm["spmv_launches"] / 1e3
    peak, peak_kind = load_peaks()
    achieved = tm["spmv_bytes"] / spmv_avg_s / 1e9
    # the symmetric product with coded indices reports fewer bytes than the one
    # with 4-byte columns and lower references (stencil-like patterns)
    upper_b, lower_b = (info["nnzb"] + p.n_nodes) // 2, (info["nnzb"] - p.n_nodes) // 2
    coded = sym and tm["spmv_bytes"] != upper_b * 40 + lower_b * 8 + 8 * info["n_dof"]
    traffic = profile_traffic(("spmv_symc_fp32_192x96x96.txt" if coded else "spmv_sym_fp32_192x96x96.txt") if sym
                              else "spmv_sell_fp32_192x96x96.txt")
    full_bytes32 = 40 * info["nnzb"] + 4 * (p.n_nodes + 1) + 8 * info["n_dof"]  # full block-CSR product, FP32

    # ---- plain FP64 PCG on the same mesh
    m.solve(b, fp64, x=x)
    f_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.fp64_steps + 1)]
    f_ev[0].record(stream)
    fst = None
    for k in range(args.fp64_steps):
        _, fst = m.solve(b, fp64, x=x)
        f_ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    t_fp64 = max_over_ranks(sum(f_ev[k].elapsed_time(f_ev[k + 1]) for k in range(args.fp64_steps))
                            / args.fp64_steps / 1e3, dev)
    u_fp64 = x.clone()
    m.set_instrument(True)
    m.solve(b, fp64, x=x)
    tm64 = m.last_timing()
    m.set_instrument(False)
    achieved64 = tm64["spmv_bytes"] / (tm64["spmv_ms"] / tm64["spmv_launches"] / 1e3) / 1e9
    du = (torch.linalg.vector_norm(u_mixed - u_fp64) / torch.linalg.vector_norm(u_fp64)).item()
    _, vm_m = m.stress(u_mixed, want_sigma=False)
    _, vm_f = m.stress(u_fp64, want_sigma=False)
    dvm = (torch.max(torch.abs(vm_m - vm_f)) / torch.max(torch.abs(vm_f))).item()

    # ---- end to end through the C-ABI with pinned host buffers (copies timed)
    b_pin = torch.from_numpy(b_host).pin_memory()
    x_pin = torch.zeros_like(b_pin).pin_memory()
    m.solve(b_pin, mixed, x=x_pin)  # staging pool warm-up
    e_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier(dev)
    e_ev[0].record(stream)
    e_steps = args.steps
    for _ in range(e_steps):
        _, est = m.solve(b_pin, mixed, x=x_pin)
    e_ev[1].record(stream)
    torch.cuda.synchronize(dev)
    t_e2e = max_over_ranks(e_ev[0].elapsed_time(e_ev[1]) / e_steps / 1e3, dev)

    # ---- multigrid-preconditioned PCG on the same mesh: FP32 V-cycle inside FP64 PCG
    mg_line = None
    if not args.no_extras:
        try:
            nx, ny, nz = mesh_dims(args.mesh)
            # a throwaway hierarchy on an 8x4x4 box first, so that the set-up time
            # below does not carry the process's first launches of the multigrid kernels
            w = ufc.FemModel.from_problem(ufc.mesh.cantilever(8, 4, 4, 8.0, 4.0, 4.0), device=local)
            w.assemble(ufc.BUILD_FP64)
            w.mg_setup(8, 4, 4, precision=ufc.PRECISION_FP32_REFINE)
            w.solve(ufc.lifted_rhs(w, w.problem.f), ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG))
            w.close()
            lv, cdof, setup_ms = m.mg_setup(nx, ny, nz, precision=ufc.PRECISION_FP32_REFINE)
            mga = ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG)
            m.solve(b, mga, x=x)
            ts, mst = [], None
            for _ in range(3):
                g_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                g_ev[0].record(stream)
                _, mst = m.solve(b, mga, x=x)
                g_ev[1].record(stream)
                torch.cuda.synchronize(dev)
                ts.append(g_ev[0].elapsed_time(g_ev[1]) / 1e3)
            u_mg = x.clone()
            mg_line = {"value": max_over_ranks(statistics.median(ts), dev), "unit": UNIT, "iters": mst.niter,
                       "rnorm": mst.rnorm, "levels": lv, "coarsest_dof": cdof, "setup_s": setup_ms / 1e3,
                       "u_rel_l2_vs_fp64_jacobi": (torch.linalg.vector_norm(u_mg - u_fp64)
                                                    / torch.linalg.vector_norm(u_fp64)).item(),
                       "solver": "PCG (FP64 matrix, vectors, residual) with a geometric multigrid V-cycle in FP32: "
                                 "Galerkin coarse boxes, Chebyshev degree 2 on D^-1 A, dense coarsest inverse; "
                                 "set-up (hierarchy) outside the timed solve, like the assembly; setup_s timed "
                                 "after a throwaway 8x4x4 set-up (first kernel launches excluded)"}
        except Exception as e:  # a failure here must not lose the headline line
            mg_line = {"error": f"{type(e).__name__}: {e}"}

    # ---- the other storage on the same mesh, one solve of each path
    other = None
    if sym:
        m.assemble(ufc.BUILD_FP64 | ufc.BUILD_FP32_ROUNDED)
        o = {}
        for key, algo in (("mixed", mixed), ("fp64", fp64)):
            m.solve(b, algo, x=x)
            o_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            o_ev[0].record(stream)
            _, ost = m.solve(b, algo, x=x)
            o_ev[1].record(stream)
            torch.cuda.synchronize(dev)
            o[key] = max_over_ranks(o_ev[0].elapsed_time(o_ev[1]) / 1e3, dev)
            o[key + "_iters"] = ost.niter
        m.set_instrument(True)
        m.solve(b, mixed, x=x)
        tmf = m.last_timing()
        m.set_instrument(False)
        f_us = tmf["spmv_ms"] / tmf["spmv_launches"] * 1e3
        other = {"storage": "full SELL-32 block CSR", "value": o["mixed"], "iters": o["mixed_iters"],
                 "fp64_value": o["fp64"], "fp64_iters": o["fp64_iters"], "unit": UNIT,
                 "spmv_us": f_us, "spmv_achieved_gbs": tmf["spmv_bytes"] / f_us / 1e3,
                 "spmv_frac": tmf["spmv_bytes"] / f_us / 1e3 / peak,
                 "traffic": profile_traffic("spmv_sell_fp32_192x96x96.txt")}

    cpu = None
    oracle_acc = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        gpu_sols = {"fp32_refine": u_mixed, "fp64": u_fp64}
        if mg_line and "value" in mg_line:
            gpu_sols["multigrid"] = u_mg
        sols = {k: v.cpu().numpy() for k, v in gpu_sols.items()}
        vms = {k: m.stress(v, want_sigma=False)[1].cpu().numpy() for k, v in gpu_sols.items()}
        cpu, oracle_acc = oracle_reference(p, sols, vms, gpu_csr=lambda: m.csr_export(index_base=0)[:3])
        del sols, vms

    mean = lambda xs: sum(xs) / len(xs)  # noqa: E731
    csr64_bytes = 12 * info["nnz"] + 4 * (info["n_dof"] + 1) + 16 * info["n_dof"] + 88 * info["n_dof"]
    fp64_csr_s = csr64_bytes / (peak * 1e9) * fst.niter
    line = {
        "metric": METRIC, "value": t_mixed, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed * 1e3,
        "speedup_vs_fp64": t_fp64 / t_mixed,
        "fp64_path": {"value": t_fp64, "unit": UNIT, "iters": fst.niter, "rnorm": fst.rnorm,
                      "spmv_achieved_gbs": achieved64,
                      "dof_iterations_per_s": world * info["n_dof"] * fst.niter / t_fp64},
        "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (matrix, CG vectors, SpMV rows) + f64 (solution, residual replacement)",
        "data": "synthetic (seeded numpy mesh and moduli)",
        "config": {"workload": workload(args.mesh), "mesh": args.mesh, "n_dof": info["n_dof"], "nnz": info["nnz"],
                   "nnzb": info["nnzb"], "sell_blocks": info["sell_blocks"],
                   "parallelism": "replicas" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (FP32 matrix 1.0 GB symmetric / 1.93 GB full per SpMV)",
                   "storage": args.storage,
                   "solver": "Jacobi-PCG, FP32 SELL-BSR3 matrix rounded from FP64 assembly"
                             + (", symmetric half storage" if sym else "")
                             + ", FP32 vectors and row sums, FP64 x, FP64 matrix-free residual replacement "
                               "(delta 0.1); the FP64 path uses the same storage"},
        "iters": mean([s.niter for s in states]), "refinements": mean([s.n_refine for s in states]),
        "rnorm": max(s.rnorm for s in states),
        "dof_iterations_per_s": world * info["n_dof"] * mean([s.niter for s in states]) / t_mixed,
        "fp64_scalar_csr_equivalent": {
            "value": fp64_csr_s, "unit": UNIT, "speedup": fp64_csr_s / t_mixed,
            "model": "the reference's FP64 scalar CSR form (RT_CSRMatrix_matvec: 12 nnz + 4 (n+1) + 16 n bytes per "
                     "SpMV) plus FP64 vector updates (88 B/DOF) at the measured copy peak, times this run's FP64 "
                     "iteration count: a floor for that storage on this GPU, a secondary figure, not the headline"},
        "accuracy_vs_fp64_gpu": {"u_rel_l2": du, "von_mises_rel_max": dvm},
        "assembly": {"pattern_ms": pattern_ms, "fp64_plus_rounded_fp32_ms": asm_ms, "fp32_element_ms": asm32_ms,
                     "with_storage_ms": build_ms,
                     "elements_per_s_fp32": p.n_elems / (asm32_ms / 1e3), "host_setup_s": setup_s},
        "roofline": {"bound": "hbm",
                     "kernel": ("k_spmv_symc<float,float,float,kCg> (symmetric SELL-32 BSR3 SpMV, coded indices: "
                                "16 + 16 code bytes per row, + p.Ap)" if coded else
                                "k_spmv_sym<float,float,float,kCg> (symmetric SELL-32 BSR3 SpMV + p.Ap)" if sym else
                                "k_spmv<float,float,float,kCg> (SELL-32 BSR3 SpMV + p.Ap)"),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": tm["spmv_bytes"], "avg_launch_us": spmv_avg_s * 1e6,
                     "launches_timed": tm["spmv_launches"],
                     "full_storage_bytes_per_launch": full_bytes32,
                     "full_storage_equivalent_gbs": full_bytes32 / spmv_avg_s / 1e9},
        "e2e": {"value": t_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * p.n_dof, "d2h_bytes_per_step": 8 * p.n_dof,
                "api": "ufc_pcg_solve(mem=UFC_MEM_HOST) via FemModel.solve on pinned host buffers"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if oracle_acc:
        # the GPU solutions against the oracle's own solve of the same problem
        oracle_acc["target_u_rel_l2"] = 1e-9
        oracle_acc["note"] = ("u_rel_l2 = ||u - u_oracle|| / ||u_oracle||, u_rel_max = max|u - u_oracle| / "
                              "max|u_oracle|, von_mises_rel_max = max over Gauss points |vm - vm_oracle| / max "
                              "vm_oracle, residual_rel = ||b - K u|| / ||b|| with the oracle's canonical CSR and lifted b")
        line["accuracy_vs_oracle"] = oracle_acc
    if other:
        line["other_storage"] = other
    if mg_line:
        line["multigrid"] = mg_line
    if cpu:
        line["cpu_baseline"] = cpu
    if not args.no_extras and world == 1:
        m.close()
        line["other_configs"] = other_configs(ufc, local, stream, cpu=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    m.close()
    if dist:
        import torch.distributed as td

        td.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
