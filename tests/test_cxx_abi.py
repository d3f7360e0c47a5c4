"""The reference-signature C++ entry points (OS_SART, CG, evalProjBack over
thrust::host_vector, include/ctlab_b200_recon.hpp) link into C++ callers built
by the host compiler and by nvcc for sm_100a (thrust's ABI namespace differs
between the two, so the library exports both).  Link only: no GPU needed."""
import os
import shutil
import subprocess

import pytest

from ctlab_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "recon_caller.cpp")
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")), "include")


def build_caller(compiler: str, out: str) -> None:
    libdir = os.path.dirname(_lib.LIB_PATH)
    common = ["-std=c++17", "-I" + os.path.join(ROOT, "include"), SRC, "-L" + libdir, "-lctlab_b200",
              "-Xlinker", "-rpath=" + libdir, "-o", out]
    if compiler == "host":
        cmd = [shutil.which("g++") or "g++", "-I" + CUDA_INC] + common
    else:
        cmd = ["nvcc", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a"] + common
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("compiler", ["host", "nvcc"])
def test_cxx_caller_links_against_reference_signatures(compiler, tmp_path):
    build_caller(compiler, str(tmp_path / "caller"))
    assert os.path.exists(tmp_path / "caller")


def test_library_exports_cxx_entry_points_for_both_thrust_abis():
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for name in ("OS_SART(thrust::", "CG(thrust::"):
        lines = [l for l in out.splitlines() if name in l]
        assert len(lines) == 2, lines  # nvcc sm_100a namespace and host-compiler namespace
    assert "evalProjBack(bool, ForwardDDMethod, BackwardDDMethod)" in out
