"""The C-ABI library loads, exports every function include/ufc_gpu.h declares,
and its structs have the sizes and field offsets the ctypes mirror assumes
(checked against the C compiler's view of the header).  No GPU needed: compute
entry points are not called, and context creation without a device returns
IF_STATUS_UNSUPPORTED rather than failing."""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header(pkg):
    lib = pkg.load()
    missing, extra = pkg.check_abi(lib)
    assert not missing and not extra, (missing, extra)
    assert len(pkg._abi.header_functions()) >= 25


STRUCTS = {
    "ufc_mesh_desc": "MeshDesc", "ufc_material_desc": "MaterialDesc", "ufc_bc_desc": "BcDesc",
    "ufc_pattern_info": "PatternInfo", "ufc_csr_export_arg": "CsrExportArg", "ufc_elem_ke_arg": "ElemKeArg",
    "ufc_elem_fe_arg": "ElemFeArg", "ufc_mat_update_arg": "MatUpdateArg", "ufc_solver_algo": "SolverAlgo",
    "ufc_solver_state": "SolverState", "ufc_nr_arg": "NrArg", "ufc_timing_info": "TimingInfo",
    "ufc_step_arg": "StepArg", "ufc_face_load_arg": "FaceLoadArg", "ufc_mg_arg": "MgArg",
}


def test_struct_layouts_match_c(pkg, tmp_path):
    A = pkg._abi
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT}/include/ufc_gpu.h"', "int main(void){"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in getattr(A, pyname)._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for cname, pyname in STRUCTS.items():
        S = getattr(A, pyname)
        assert int(got[cname]) == C.sizeof(S), cname
        for fname, _ in S._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(S, fname).offset, f"{cname}.{fname}"


def test_status_codes_match_header(pkg):
    text = open(os.path.join(ROOT, "include", "ufc_gpu.h")).read()
    A = pkg._abi
    for name in ["OK", "INVALID", "ERROR", "CONVERGED", "NOT_CONVERGED", "NOT_FOUND", "WARN", "MEM_ERROR",
                 "IO_ERROR", "EXISTS", "FATAL", "UNSUPPORTED"]:
        assert f"#define UFC_STATUS_{name} {getattr(A, 'STATUS_' + name)}" in text


def test_context_without_device_reports_status(pkg):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; covered by the GPU tests")
    lib = pkg.load()
    h = C.c_void_p()
    assert lib.ufc_ctx_create(0, C.byref(h)) == pkg._abi.STATUS_UNSUPPORTED
    assert lib.ufc_ctx_destroy(None) == pkg._abi.STATUS_INVALID
    with pytest.raises(pkg.UfcError) as ei:
        pkg.FemModel()
    assert ei.value.status_code == pkg._abi.STATUS_UNSUPPORTED


def test_missing_library_fails_loudly(pkg, tmp_path):
    with pytest.raises(pkg.LibraryMissing):
        pkg._abi.load(str(tmp_path / "nope.so"))
