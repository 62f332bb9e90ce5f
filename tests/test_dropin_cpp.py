"""The C++ drop-in headers (include/elemgpu/elemental.hpp) compile against the
reference's API shape and, on a GPU, pass a driver written like the
reference's own tests/lapack-like/{Cholesky,SequentialLU}.cpp."""
import os
import subprocess

import pytest

import elemental_b200 as eg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_test.cpp")


def _build(tmp_path):
    eg.lib()  # make sure the library exists
    exe = str(tmp_path / "dropin_test")
    libdir = os.path.dirname(eg.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-L", libdir,
           "-lelemgpu", f"-Wl,-rpath,{libdir}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_dropin_headers_compile(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_dropin_driver_on_gpu(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "PASSED" in out.stdout
