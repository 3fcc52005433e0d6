"""Where the extra iterations of the refined FP32 solve come from, on the CPU.

Jacobi-PCG with residual replacement (the FP32_REFINE schedule: replace the
recursive residual by the FP64 b - K x whenever it has fallen by 0.1) on the
oracle's assembly of a 16x8x8 lognormal cantilever:
  - FP64 everywhere, with or without replacement: the FP64 count;
  - CG on the FP32-rounded matrix with its own residual: the FP64 count too;
  - FP32 matrix in the recursion but FP64 replacement residuals, or FP64 matrix
    with FP32 vectors: about 40 % more iterations.
The surplus comes from running the recursion with an operator (or vectors)
rounded to FP32 while converging to the FP64 system, which each replacement
corrects only to about kappa * 2^-24; it is a property of the method, not of
the kernels."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def system(pkg, orc):
    sp = pytest.importorskip("scipy.sparse")
    p = pkg.mesh.lognormal_cantilever(16, 8, 8, 4)
    m = orc.Model(p)
    K = m.assemble()
    A64 = sp.csr_matrix((K.val, K.col, K.row_ptr), shape=(K.n, K.n))
    return A64, m.lifted_rhs()


def _pcg(A_rec, A_res, b, vdt, replace, delta=0.1, rtol=1e-10, max_iter=5000):
    """Jacobi-PCG whose recursion uses A_rec and vectors of type vdt; the
    solution accumulates in FP64 and replacements use r = b - A_res x."""
    d = A_res.diagonal()
    dinv = (1.0 / d).astype(vdt)
    tol = rtol * np.linalg.norm(b)
    x = np.zeros(b.size)
    r = b.astype(vdt)
    z = dinv * r
    p = z.copy()
    rz = float(np.dot(r, z))
    rr_ref = float(np.dot(r, r))
    for it in range(1, max_iter + 1):
        q = (A_rec @ p.astype(A_rec.dtype)).astype(vdt)
        alpha = rz / float(np.dot(p.astype(np.float64), q))
        x += alpha * p
        r = (r - vdt(alpha) * q).astype(vdt)
        z = dinv * r
        rz_new = float(np.dot(r.astype(np.float64), z))
        rr = float(np.dot(r.astype(np.float64), r))
        if rr <= tol * tol or (replace and rr < delta * delta * rr_ref):
            res = b - A_res @ x
            if np.linalg.norm(res) <= tol:
                return it
            if replace:
                r = res.astype(vdt)
                z = dinv * r
                rz_new = float(np.dot(r.astype(np.float64), z))
                rr_ref = float(np.dot(r.astype(np.float64), r))
        p = (z + vdt(rz_new / rz) * p).astype(vdt)
        rz = rz_new
    return max_iter + 1


def test_fp32_iteration_surplus_comes_from_the_operator_mismatch(system):
    A64, b = system
    A32 = A64.astype(np.float32)
    A32d = A32.astype(np.float64)
    n64 = _pcg(A64, A64, b, np.float64, replace=False)
    n64_rep = _pcg(A64, A64, b, np.float64, replace=True)
    n32_own = _pcg(A32d, A32d, b, np.float64, replace=False)
    n32_mat = _pcg(A32d, A64, b, np.float64, replace=True)
    n32_vec = _pcg(A64, A64, b, np.float32, replace=True)
    n32_all = _pcg(A32, A64, b, np.float32, replace=True)
    assert n64 < 5000
    # replacement alone and the FP32 matrix on its own cost nothing
    assert abs(n64_rep - n64) <= 0.02 * n64
    assert abs(n32_own - n64) <= 0.02 * n64
    # mixing the FP32 recursion with FP64 residuals costs about 40 %
    for n in (n32_mat, n32_vec, n32_all):
        assert 1.2 * n64 < n < 1.8 * n64, (n64, n32_mat, n32_vec, n32_all)
