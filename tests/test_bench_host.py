"""Host-side parts of bench.py on the CPU: the oracle sample's residual check
and its comparison of an exported CSR with the oracle's assembly."""
import numpy as np


def test_cpu_sample_residuals_and_csr_comparison(pkg, orc):
    import bench

    p = pkg.mesh.lognormal_cantilever(6, 3, 3, seed=4)
    K = orc.Model(p).assemble()
    exact = lambda: (K.row_ptr.copy(), K.col.copy(), K.val * (1.0 + 2.0 ** -52))  # noqa: E731
    setup, per, threads, res = bench.cpu_sample(p, 3, check={"zero": np.zeros(p.n_dof)}, gpu_csr=exact)
    assert setup >= 0.0 and len(per) == 1 and per[0] > 0.0 and threads >= 1
    assert abs(res["zero"] - 1.0) < 1e-12  # ||b - K 0|| / ||b||
    csr = res["csr"]
    assert csr["pattern_equal"] and csr["nnz"] == K.col.size
    assert 0.0 < csr["values_rel_max_err"] <= 1e-15

    def shifted():
        col = K.col.copy()
        col[0] = (col[0] + 1) % p.n_dof
        return K.row_ptr.copy(), col, K.val.copy()

    _, _, _, res = bench.cpu_sample(p, 1, gpu_csr=shifted)
    assert res["csr"]["pattern_equal"] is False and res["csr"]["values_rel_max_err"] is None


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
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "8x4x4" in d["config"]["workload"]
