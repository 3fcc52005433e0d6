"""The allocation-free SpMV entry point, through the C-ABI.

ufc_csr_spmv_dot_noalloc serves callers that cannot allocate device memory (a
host code whose device memory all comes from its own fixed pool, or one that
may not enter the CUDA allocator on its hot path): its dot-product scratch is a
static device array.  This test checks it on two calls in a row, which also
exercises the shared scratch being reused, against the existing entry point
ufc_spmv (same matrix, exported to device memory) and against the oracle's
CSR product, within the SpMV tolerance of the other parity tests (1e-13
relative), on a small mesh and on one of 143,811 rows whose 562 blocks all
reduce through the last-block election.  It lives in its own file, collected
last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 16777216


@pytest.mark.parametrize("shape", [(10, 6, 5), (56, 28, 28)])
def test_csr_spmv_dot_noalloc_matches_ufc_spmv_and_oracle(pkg, orc, shape):
    torch = pytest.importorskip("torch")
    A = pkg._abi
    p = pkg.mesh.lognormal_cantilever(*shape, seed=9)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    n, nnz = m.info.n_dof, m.info.nnz
    dev = torch.device("cuda", 0)
    rp = torch.empty(n + 1, dtype=torch.int64, device=dev)
    col = torch.empty(nnz, dtype=torch.int32, device=dev)
    val = torch.empty(nnz, dtype=torch.float64, device=dev)
    arg = A.CsrExportArg(0, A.MEM_DEVICE, rp.data_ptr(), col.data_ptr(), val.data_ptr(), None)
    assert m.lib.ufc_csr_export(m.h, C.byref(arg)) == 0
    K = orc.Model(p).assemble()  # the oracle's canonical CSR of the same problem
    lib = m.lib
    stream = torch.cuda.current_stream(dev)
    err = C.create_string_buffer(256)
    rng = np.random.default_rng(5)
    for call in range(2):
        x_h = rng.standard_normal(n)
        x = torch.from_numpy(x_h).to(dev)
        y = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        xy = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        st = lib.ufc_csr_spmv_dot_noalloc(n, rp.data_ptr(), col.data_ptr(), val.data_ptr(), x.data_ptr(),
                                          y.data_ptr(), xy.data_ptr(), C.c_void_p(stream.cuda_stream), err, 256)
        assert st == 0, err.value
        y_ref = m.spmv(x)  # existing entry point ufc_spmv (SELL storage, FP64)
        torch.cuda.synchronize(dev)
        scale = torch.max(torch.abs(y_ref)).item()
        assert torch.max(torch.abs(y - y_ref)).item() <= 1e-13 * scale, call
        dot_ref = torch.dot(x, y_ref).item()
        assert abs(xy.item() - dot_ref) <= 1e-13 * torch.dot(torch.abs(x), torch.abs(y_ref)).item(), call
        # the oracle's product of the same matrix on the CPU
        y_o = K.matvec(x_h)
        y_h = y.cpu().numpy()
        assert np.abs(y_h - y_o).max() <= 1e-13 * np.abs(y_o).max(), call
        assert abs(xy.item() - float(np.dot(x_h, y_o))) <= 1e-13 * float(np.dot(np.abs(x_h), np.abs(y_o))), call
    # sizes beyond the static scratch are rejected with a clear message
    st = lib.ufc_csr_spmv_dot_noalloc(MAX_ROWS + 1, rp.data_ptr(), col.data_ptr(), val.data_ptr(), x.data_ptr(),
                                      y.data_ptr(), xy.data_ptr(), C.c_void_p(stream.cuda_stream), err, 256)
    assert st == A.STATUS_INVALID and b"UFC_NOALLOC_MAX_ROWS" in err.value
    m.close()
