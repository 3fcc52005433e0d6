"""A C program drives the C-ABI the way the reference's Fortran would (through
include/ufc_gpu_brg.f90): tests/c/ufc_c_drop_in.c, built with gcc against
include/ufc_gpu.h and libufc_gpu.so only.  Without a device it must stop at
context creation with IF_STATUS_UNSUPPORTED (exit 77); on a B200 it runs the
linear static, multigrid and J2 step sequences end to end."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ufc-fem-kernel_b200")


def _build(tmp_path):
    exe = tmp_path / "ufc_c_drop_in"
    subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "ufc_c_drop_in.c"), "-L", LIBDIR, "-lufc_gpu",
                    f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", str(exe)], check=True)
    return exe


def test_c_caller_builds_and_fails_loudly_without_device(pkg, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU test runs the program")
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 77, (r.returncode, r.stdout, r.stderr)
    assert "IF_STATUS_UNSUPPORTED" in r.stdout


@pytest.mark.gpu
def test_c_caller_end_to_end(pkg, tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "C drop-in OK" in r.stdout
