"""Host-side parts of bench.py on the CPU: the oracle reference solve with its
error figures and its comparison of an exported CSR with the oracle's
assembly, and the reference arm's JSON line."""
import numpy as np


def test_oracle_reference_errors_and_csr_comparison(pkg, orc):
    """bench.oracle_reference: the oracle's own solve gives the measured CPU
    time and the reference solution; a planted error in a 'GPU' solution (here
    a CPU copy) shows in its displacement and von Mises errors, and an exact
    copy reads zero."""
    import bench

    p = pkg.mesh.lognormal_cantilever(6, 3, 3, seed=4)
    model = orc.Model(p)
    K = model.assemble()
    u, info = orc.pcg(K, model.lifted_rhs(), rtol=1e-14)
    bad = u.copy()
    bad[np.argmax(np.abs(u))] *= 1.0 + 1e-6  # planted on the CPU
    vm = {"exact": model.elastic_vm(u)[1], "bad": model.elastic_vm(bad)[1]}
    exact = lambda: (K.row_ptr.copy(), K.col.copy(), K.val * (1.0 + 2.0 ** -52))  # noqa: E731
    cpu, acc = bench.oracle_reference(p, {"exact": u, "bad": bad}, vm, gpu_csr=exact)
    assert cpu["value"] > 0.0 and cpu["kind"] == "port" and cpu["cores"] >= 1 and "whole" in cpu["sample"]
    assert acc["exact"]["u_rel_l2"] < 1e-12 and acc["exact"]["von_mises_rel_max"] < 1e-12
    assert acc["exact"]["residual_rel"] < 1e-12
    assert 1e-8 < acc["bad"]["u_rel_max"] <= 1.01e-6 and acc["bad"]["von_mises_rel_max"] > 1e-9
    assert acc["oracle_rtol_1e-10"]["residual_rel"] <= 1e-10
    assert acc["reference"]["true_residual_rel"] < acc["oracle_rtol_1e-10"]["residual_rel"]
    csr = acc["csr"]
    assert csr["pattern_equal"] and csr["nnz"] == K.col.size
    assert 0.0 < csr["values_rel_max_err"] <= 1e-15

    def shifted():
        col = K.col.copy()
        col[0] = (col[0] + 1) % p.n_dof
        return K.row_ptr.copy(), col, K.val.copy()

    _, acc = bench.oracle_reference(p, gpu_csr=shifted)
    assert acc["csr"]["pattern_equal"] is False and acc["csr"]["values_rel_max_err"] is None


def test_reference_arm_json_line():
    """`bench.py --impl reference` (the oracle's CPU Jacobi-PCG) prints one JSON
    line with the contract's keys, on a small mesh so that it runs in seconds."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--mesh", "8x4x4",
                          "--steps", "1", "--warmup", "1"], check=True, capture_output=True, text=True,
                         cwd=root, timeout=600).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "s" and d["value"] > 0.0 and d["higher_is_better"] is False
    assert d["steps"] == 1 and d["steps_requested"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert "whole" in d["cpu_baseline"]["sample"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "8x4x4" in d["config"]["workload"]
