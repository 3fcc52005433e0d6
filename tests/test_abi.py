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


def _f90_types(text):
    """Components (name, kind) of every TYPE, BIND(C) in the Fortran bridge, in order."""
    import re

    types, cur = {}, None
    for raw in text.split("\n"):
        line = raw.split("!")[0].strip()
        m = re.match(r"TYPE,\s*BIND\(C\),\s*PUBLIC\s*::\s*(\w+)", line, re.I)
        if m:
            cur = m.group(1).lower()
            types[cur] = []
            continue
        if cur and re.match(r"END\s+TYPE", line, re.I):
            cur = None
            continue
        if cur and "::" in line:
            kind, names = (part.strip() for part in line.split("::", 1))
            names = re.sub(r"=\s*[^,]+", "", names)  # default initialisations
            for nm in names.split(","):
                nm = nm.strip()
                dim = re.match(r"(\w+)\((\d+)\)", nm)
                types[cur].append((dim.group(1) if dim else nm, kind.upper().replace(" ", ""),
                                   int(dim.group(2)) if dim else 1))
    return types


def test_fortran_bridge_covers_the_header(pkg):
    """include/ufc_gpu_brg.f90 (not compiled here: no Fortran compiler) binds
    every function of the header, its BIND(C) types list the fields of the C
    structs in order with matching kinds, and its constants have the header's
    values."""
    import re

    A = pkg._abi
    f90 = open(os.path.join(ROOT, "include", "ufc_gpu_brg.f90")).read()
    header = open(os.path.join(ROOT, "include", "ufc_gpu.h")).read()
    bound = {n.lower() for n in re.findall(r"BIND\(C,\s*NAME\s*=\s*'(ufc_\w+)'\)", f90, flags=re.I)}
    assert set(A.header_functions()) <= bound, sorted(set(A.header_functions()) - bound)
    kinds = {"INTEGER(C_INT32_T)": (C.c_int32,), "INTEGER(C_INT64_T)": (C.c_int64,),
             "REAL(C_DOUBLE)": (C.c_double,), "TYPE(C_PTR)": (C.c_void_p,)}
    types = _f90_types(f90)
    for cname, pyname in STRUCTS.items():
        assert cname in types, cname
        fields = getattr(A, pyname)._fields_
        comps = types[cname]
        assert [c[0].lower() for c in comps] == [f[0].lower() for f in fields], cname
        for (nm, kind, dim), (_, ctype) in zip(comps, fields):
            if kind.startswith("TYPE(UFC_"):
                assert ctype.__name__ == STRUCTS[kind[5:-1].lower()], (cname, nm)
            elif dim > 1:
                assert issubclass(ctype, C.Array) and ctype._length_ == dim, (cname, nm)
            elif kind == "TYPE(C_PTR)":
                assert ctype is C.c_void_p or issubclass(ctype, C._Pointer) or ctype in (C.c_char_p,), (cname, nm)
            else:
                assert C.sizeof(ctype) == C.sizeof(kinds[kind][0]) and (ctype in (C.c_double,)) == (
                    kinds[kind][0] is C.c_double), (cname, nm, kind)
    defines = dict(re.findall(r"#define (UFC_\w+) (-?\d+)", header))
    params = re.findall(r"\b(UFC_\w+)\s*=\s*(-?\d+)", f90)
    assert len(params) >= 30
    for name, value in params:
        assert name in defines and int(defines[name]) == int(value), name
