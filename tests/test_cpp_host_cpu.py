"""The C++ host layer (include/pimc_b200.hpp) without a GPU: it compiles with
-Wall -Wextra -Werror against the C ABI, links against libpimc_b200.so, and
a PathData on a machine without a usable device raises pimc_b200::Error
carrying PIMC_E_CUDA."""
import os
import shutil
import subprocess

import pytest

from helpers import ROOT

LIBDIR = os.path.join(ROOT, "pimcplusplus_b200")
INCLUDE = os.path.join(ROOT, "include")


def build_host_check(out_dir):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    exe = os.path.join(str(out_dir), "host_cpp_check")
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", INCLUDE,
                    os.path.join(ROOT, "tests", "host_cpp_check.cc"), "-o", exe, "-L", LIBDIR, "-lpimc_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_cpp_host_layer_builds_and_reports_missing_device(tmp_path):
    exe = build_host_check(tmp_path)
    out = subprocess.run([exe, "cpu"], capture_output=True, text=True, timeout=120, check=True).stdout.split()
    assert out[0] in ("created", "error")
    if out[0] == "error":
        assert int(out[1]) == 2  # PIMC_E_CUDA
