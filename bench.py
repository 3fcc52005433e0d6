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
here) on the host cores: each step is a bounded sample of CG iterations on the
same matrix, extrapolated to the iteration count of FP64 Jacobi-PCG on this
mesh.
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
# FP64 Jacobi-PCG on the 192x96x96 lognormal cantilever reaches rtol 1e-10 in
# 3151 iterations (measured on a B200 with this repository's FP64 path; the
# oracle runs the same recurrences).  Used to extrapolate the CPU samples.
FP64_ITERS_192x96x96 = 3151
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
    ap.add_argument("--cpu-iters", type=int, default=12, help="CG iterations per CPU sample")
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


def cpu_sample(p, iters, reps=1, check=None, gpu_csr=None):
    """Oracle (CPU FP64, all host threads) per-iteration time of Jacobi-PCG on the
    problem's canonical CSR: setup time, seconds per iteration, threads, and for
    each GPU solution in `check` (name -> host array) its relative residual
    ||b - K u|| / ||b|| with the oracle's own assembly and right-hand side.
    gpu_csr, when given, returns the GPU's exported canonical CSR (row_ptr, col,
    FP64 values), compared with the oracle's: pattern equality and the largest
    value difference relative to the largest entry (under "csr")."""
    from oracle import oracle as O

    import numpy as np

    t0 = time.perf_counter()
    model = O.Model(p)
    K = model.assemble()
    b = model.lifted_rhs()
    setup = time.perf_counter() - t0
    csr = None
    if gpu_csr is not None:
        rp, col, v = gpu_csr()
        same = bool(np.array_equal(rp, K.row_ptr) and np.array_equal(col, K.col))
        csr = {"pattern_equal": same, "nnz": int(col.size),
               "values_rel_max_err": float(np.abs(v - K.val).max() / np.abs(K.val).max()) if same else None}
        del rp, col, v
    per = []
    for _ in range(reps):
        t = time.perf_counter()
        O.pcg(K, b, max_iter=-iters)
        per.append((time.perf_counter() - t) / iters)
    bn = float(np.linalg.norm(b))
    res = {k: float(np.linalg.norm(b - K.matvec(u)) / bn) for k, u in (check or {}).items()}
    if csr is not None:
        res["csr"] = csr
    return setup, per, O.num_threads(), res


def cpu_linear(p, iters_gpu, full_max_dof=50000, sample_iters=12):
    """The oracle's FP64 Jacobi-PCG (CPU, all host threads) on one linear-elastic
    problem: the whole solve to rtol 1e-10 when the problem has at most
    full_max_dof DOF, else sample_iters iterations extrapolated to the GPU's FP64
    iteration count; the CSR assembly is timed on its own."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    model = O.Model(p)
    K = model.assemble()
    b = model.lifted_rhs()
    t_asm = time.perf_counter() - t0
    if p.n_dof <= full_max_dof:
        t = time.perf_counter()
        _, info = O.pcg(K, b, rtol=1e-10)
        s, sample = time.perf_counter() - t, f"the whole solve ({info['iters']} iterations)"
    else:
        t = time.perf_counter()
        O.pcg(K, b, max_iter=-sample_iters)
        per = (time.perf_counter() - t) / sample_iters
        s, sample = per * iters_gpu, f"{sample_iters} iterations, {per * 1e3:.1f} ms/iter x {iters_gpu} (GPU FP64 count)"
    return {"s": s, "kind": "port", "cores": O.num_threads(), "assembly_s": t_asm, "sample": sample}


def linear_static(ufc, local, p, cpu=False):
    """Time-to-rtol 1e-10 of one linear-elastic problem from x0 = 0: FP64
    Jacobi-PCG, the FP32+FP64-refined one (full storage) and FP64 PCG with the
    multigrid preconditioner, each timed by the library's CUDA events after one
    warm-up solve, with the assembly time."""
    import torch

    dev = torch.device("cuda", local)
    m = ufc.FemModel.from_problem(p, device=local)
    ka = m.assemble(ufc.BUILD_FP64 | ufc.BUILD_FP32_ROUNDED)
    b = torch.from_numpy(ufc.lifted_rhs(m, p.f)).to(dev)
    x = torch.zeros_like(b)
    res = {"n_dof": p.n_dof, "elements": p.n_elems, "assembly_ms": ka}
    for key, pm in (("fp64", ufc.PRECISION_FP64), ("fp32_refine", ufc.PRECISION_FP32_REFINE)):
        a = ufc.SolverAlgo(tolerance=1e-10, precision_mode=pm)
        x.zero_()
        m.solve(b, a, x=x, raise_on_not_converged=False)
        x.zero_()
        _, st = m.solve(b, a, x=x, raise_on_not_converged=False)
        res[key] = {"s": st.solve_time / 1e3, "iters": st.niter, "rnorm": st.rnorm, "converged": st.converged}
        if pm != ufc.PRECISION_FP64:
            res[key]["fp64_continuation_iters"] = st.fp64_iters
    # FP64 PCG with the geometric multigrid V-cycle in FP32 (set-up outside the timed solve)
    levels, coarse, setup_ms = m.mg_setup(*p.shape, precision=ufc.PRECISION_FP32_REFINE)
    a = ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG)
    x.zero_()
    m.solve(b, a, x=x, raise_on_not_converged=False)
    x.zero_()
    _, st = m.solve(b, a, x=x, raise_on_not_converged=False)
    res["multigrid"] = {"s": st.solve_time / 1e3, "iters": st.niter, "rnorm": st.rnorm, "converged": st.converged,
                        "levels": levels, "coarsest_dof": coarse, "setup_s": setup_ms / 1e3}
    m.close()
    if cpu:
        res["cpu_baseline"] = cpu_linear(p, res["fp64"]["iters"])
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


def cpu_adjoint(p, E, U, iters, sample_iters=12):
    """The oracle's cost of the 16-case adjoint workload on the CPU (all host
    threads): sample_iters FP64 Jacobi-PCG iterations on the density problem's
    stiffness extrapolated to 16 solves of the GPU block's iteration count, plus
    the sensitivity dJ/dE of all 16 cases timed in full."""
    import numpy as np

    from oracle import oracle as O

    model = O.Model(p)
    props = np.stack([E, p.props[:, 1]], axis=1)
    K = model.assemble(props=props)
    b = np.ascontiguousarray(U[0])
    t = time.perf_counter()
    O.pcg(K, b, max_iter=-sample_iters)
    per = (time.perf_counter() - t) / sample_iters
    t = time.perf_counter()
    model.adjoint_dJdE(U, U, props=props)
    t_sens = time.perf_counter() - t
    n = U.shape[0]
    return {"s": n * iters * per + t_sens, "kind": "port", "cores": O.num_threads(),
            "sample": f"{sample_iters} PCG iterations ({per * 1e3:.1f} ms/iter) x {iters} x {n} cases + "
                      f"the sensitivity of all {n} cases ({t_sens:.3f} s)"}


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
        from ufc_fem_kernel_b200.adjoint import ElasticModel

        p = ufc.mesh.config5()
        model = ElasticModel(p, device=local)
        rho = torch.tensor(p.meta["rho"], dtype=torch.float64, device=dev)
        F = torch.tensor(p.meta["F"], dtype=torch.float64, device=dev) * model.free
        model.set_moduli(210e3 * rho ** 3)
        algo = ufc.SolverAlgo(tolerance=1e-10)
        model.fem.solve_block(F, algo)  # warm-up
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        U, states = model.fem.solve_block(F, algo)
        ev[1].record(stream)
        model.fem.adjoint_sensitivity(U, U)
        ev[2].record(stream)
        torch.cuda.synchronize(dev)
        out["adjoint_128x64x64_16rhs"] = {
            "workload": "density problem 128x64x64 (E = 210e3 rho^3, rho ~ U(0.3,1)), 16 tip-load cases as one "
                        "block Jacobi-PCG to rtol 1e-10, then dJ/dE_e = -u_e.(K_e/E_e).u_e for all 16",
            "block_solve_s": ev[0].elapsed_time(ev[1]) / 1e3, "sensitivity_s": ev[1].elapsed_time(ev[2]) / 1e3,
            "iters_max": max(s.niter for s in states), "converged": all(s.converged for s in states),
            "n_dof": p.n_dof}
        # the 16 cases one after another with the multigrid preconditioner
        model.fem.mg_setup(*p.shape, precision=ufc.PRECISION_FP32_REFINE)
        mga = ufc.SolverAlgo(tolerance=1e-10, precond_type=ufc.SOLV_PREC_MG)
        Um = torch.empty_like(F)
        model.fem.solve(F[0].contiguous(), mga, x=Um[0])
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        its = []
        for k in range(F.shape[0]):
            _, sk = model.fem.solve(F[k].contiguous(), mga, x=Um[k])
            its.append(sk.niter)
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        out["adjoint_128x64x64_16rhs"]["multigrid_solves_s"] = ev[0].elapsed_time(ev[1]) / 1e3
        out["adjoint_128x64x64_16rhs"]["multigrid_iters_max"] = max(its)
        out["adjoint_128x64x64_16rhs"]["multigrid_vs_block_u_rel"] = (
            torch.linalg.vector_norm(Um - U) / torch.linalg.vector_norm(U)).item()
        # dJ/drho of case 0's compliance J = f.u against central differences
        # (h = 1e-6) on the 32 seeded elements; each difference is solved as a
        # correction K' du = f - K' u0 with the multigrid PCG
        g = model.fem.adjoint_sensitivity(U[:1].contiguous(), U[:1].contiguous()) * 3 * 210e3 * rho ** 2
        h = 1e-6
        f0 = F[0].contiguous()
        worst = 0.0
        for e in p.meta["fd_elems"]:
            d = []
            for sgn in (1.0, -1.0):
                rp = rho.clone()
                rp[int(e)] += sgn * h
                model.set_moduli(210e3 * rp ** 3)
                _, r, _, _ = model.fem.internal_force(U[0].contiguous(), f_ext=f0, update_state=False)
                du, _ = model.fem.solve(r, mga)
                d.append(torch.dot(f0, du).item())
            fd = (d[0] - d[1]) / (2 * h)
            worst = max(worst, abs(g[int(e)].item() - fd) / abs(fd))
        model.set_moduli(210e3 * rho ** 3)
        if cpu:
            out["adjoint_128x64x64_16rhs"]["cpu_baseline"] = cpu_adjoint(
                p, 210e3 * rho.cpu().numpy() ** 3, U.cpu().numpy(), max(s.niter for s in states))
        out["adjoint_128x64x64_16rhs"]["fd_check"] = {
            "elements": len(p.meta["fd_elems"]), "h": h, "max_rel_err": worst,
            "note": "adjoint dJ/drho of case 0's compliance (block solve) against central differences"}
        model.fem.close()
    except Exception as e:
        out["adjoint_128x64x64_16rhs"] = {"error": f"{type(e).__name__}: {e}"}
    return out


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
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
    samples = []
    for k in range(args.warmup + args.steps):
        t = time.perf_counter()
        O.pcg(K, b, max_iter=-args.cpu_iters)
        if k >= args.warmup:
            samples.append((time.perf_counter() - t) / args.cpu_iters)
    t_iter = statistics.median(samples)
    value = t_iter * FP64_ITERS_192x96x96
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, numpy)",
            "config": {"workload": workload(args.mesh), "parallelism": "host threads", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.cpu_iters} FP64 Jacobi-PCG iterations per step on the canonical "
                                       f"CSR (oracle, OpenMP), median s/iter x {FP64_ITERS_192x96x96} iterations; "
                                       f"CSR build {setup:.1f} s excluded"},
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
    traffic = profile_traffic("spmv_sym_fp32_192x96x96.txt" if sym else "spmv_sell_fp32_192x96x96.txt")
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
    e_steps = max(1, min(args.steps, 3))
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
                                 "set-up (hierarchy) outside the timed solve, like the assembly"}
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
    oracle_res = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        checks = {"fp32_refine": u_mixed.cpu().numpy(), "fp64": u_fp64.cpu().numpy()}
        if mg_line and "value" in mg_line:
            checks["multigrid"] = u_mg.cpu().numpy()
        setup, per, threads, oracle_res = cpu_sample(p, args.cpu_iters, check=checks,
                                                     gpu_csr=lambda: m.csr_export(index_base=0)[:3])
        iters64 = fst.niter
        cpu = {"value": per[0] * iters64, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{args.cpu_iters} FP64 Jacobi-PCG iterations of the oracle (OpenMP, canonical CSR) on "
                         f"this mesh, {per[0]*1e3:.1f} ms/iter x {iters64} iterations (this run's FP64 count); "
                         f"CPU CSR build {setup:.1f} s excluded"}

    mean = lambda xs: sum(xs) / len(xs)  # noqa: E731
    line = {
        "metric": METRIC, "value": t_mixed, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (matrix, CG vectors, SpMV rows) + f64 (solution, residual replacement)",
        "data": "synthetic (seeded numpy mesh and moduli)",
        "config": {"workload": workload(args.mesh), "mesh": args.mesh, "n_dof": info["n_dof"], "nnz": info["nnz"],
                   "nnzb": info["nnzb"], "sell_blocks": info["sell_blocks"],
                   "parallelism": "replicas" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (FP32 matrix 1.23 GB symmetric / 1.93 GB full per SpMV)",
                   "storage": args.storage,
                   "solver": "Jacobi-PCG, FP32 SELL-BSR3 matrix rounded from FP64 assembly"
                             + (", symmetric half storage" if sym else "")
                             + ", FP32 vectors and row sums, FP64 x, FP64 matrix-free residual replacement "
                               "(delta 0.1); the FP64 path uses the same storage"},
        "iters": mean([s.niter for s in states]), "refinements": mean([s.n_refine for s in states]),
        "rnorm": max(s.rnorm for s in states),
        "dof_iterations_per_s": world * info["n_dof"] * mean([s.niter for s in states]) / t_mixed,
        "fp64_path": {"value": t_fp64, "unit": UNIT, "iters": fst.niter, "rnorm": fst.rnorm,
                      "spmv_achieved_gbs": achieved64,
                      "dof_iterations_per_s": world * info["n_dof"] * fst.niter / t_fp64},
        "speedup_vs_fp64": t_fp64 / t_mixed,
        "accuracy_vs_fp64_gpu": {"u_rel_l2": du, "von_mises_rel_max": dvm},
        "assembly": {"pattern_ms": pattern_ms, "fp64_plus_rounded_fp32_ms": asm_ms, "fp32_element_ms": asm32_ms,
                     "with_storage_ms": build_ms,
                     "elements_per_s_fp32": p.n_elems / (asm32_ms / 1e3), "host_setup_s": setup_s},
        "roofline": {"bound": "hbm",
                     "kernel": ("k_spmv_sym<float,float,float,kCg> (symmetric SELL-32 BSR3 SpMV + p.Ap)" if sym else
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
    if oracle_res:
        # the GPU solutions checked with the oracle's CPU assembly of the same problem
        csr = oracle_res.pop("csr", None)
        line["accuracy_vs_oracle"] = {"residual_rel": oracle_res,
                                      "note": "||b - K u|| / ||b|| with the oracle's canonical CSR and lifted b"}
        if csr is not None:
            line["accuracy_vs_oracle"]["csr"] = csr
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
