"""The allocation-free SpMV entry point, through the C-ABI.

ufc_csr_spmv_dot_noalloc serves callers that cannot allocate device memory (a
solver loop recorded into a CUDA graph, or a host code whose device memory all
comes from its own pool): its dot-product scratch is a static device array.
This test checks it against the existing entry point ufc_spmv (same matrix,
exported to device memory) on two calls in a row, which also exercises the
shared scratch being reused, within the SpMV tolerance of the other parity
tests (1e-13 relative).  It lives in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_csr_spmv_dot_noalloc_matches_ufc_spmv(pkg):
    torch = pytest.importorskip("torch")
    A = pkg._abi
    p = pkg.mesh.lognormal_cantilever(10, 6, 5, seed=9)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    n, nnz = m.info.n_dof, m.info.nnz
    dev = torch.device("cuda", 0)
    rp = torch.empty(n + 1, dtype=torch.int64, device=dev)
    col = torch.empty(nnz, dtype=torch.int32, device=dev)
    val = torch.empty(nnz, dtype=torch.float64, device=dev)
    arg = A.CsrExportArg(0, A.MEM_DEVICE, rp.data_ptr(), col.data_ptr(), val.data_ptr(), None)
    assert m.lib.ufc_csr_export(m.h, C.byref(arg)) == 0
    lib = m.lib
    stream = torch.cuda.current_stream(dev)
    err = C.create_string_buffer(256)
    rng = np.random.default_rng(5)
    for call in range(2):
        x = torch.from_numpy(rng.standard_normal(n)).to(dev)
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
    # sizes beyond the static scratch are rejected with a clear message
    st = lib.ufc_csr_spmv_dot_noalloc(A_MAX_PLUS_ONE, rp.data_ptr(), col.data_ptr(), val.data_ptr(), x.data_ptr(),
                                      y.data_ptr(), xy.data_ptr(), C.c_void_p(stream.cuda_stream), err, 256)
    assert st == A.STATUS_INVALID and b"UFC_NOALLOC_MAX_ROWS" in err.value
    m.close()


A_MAX_PLUS_ONE = 16777216 + 1
