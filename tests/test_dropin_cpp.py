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


def _write(path, A):
    import numpy as np
    A = np.asfortranarray(A)
    with open(path, "wb") as f:
        np.array(A.shape, dtype=np.int32).tofile(f)
        A.ravel(order="F").tofile(f)


def _read(path, dtype="float64"):
    import numpy as np
    with open(path, "rb") as f:
        h, w = np.fromfile(f, dtype=np.int32, count=2)
        return np.fromfile(f, dtype=dtype, count=h * w).reshape((h, w), order="F")


@pytest.mark.gpu
def test_dropin_dist_overloads_match_oracle(tmp_path):
    """The 1 x 1 DistMatrix overloads of Cholesky (Cholesky.hpp:79-101),
    cholesky::SolveAfter (Cholesky/SolveAfter.hpp:77-134), HPDSolve
    (HPDSolve.hpp:30-41), LU (LU.hpp:220-321), lu::SolveAfter
    (LU/SolveAfter.hpp:148-195) and GaussianElimination, and Trsv
    (Trsv.hpp:20-44), through the C++ drop-in, against the oracle on the same
    inputs (tolerances of tests/test_gpu_parity.py)."""
    import numpy as np
    from elemental_b200 import inputs
    from oracle import pyoracle as orc
    exe = _build(tmp_path)
    n, k = 333, 5
    spd, ge, rhs = inputs.spd_ggt(n, 81), inputs.uniform(n, n, 82), inputs.normal(n, k, 83)
    _write(tmp_path / "spd.bin", spd)
    _write(tmp_path / "ge.bin", ge)
    _write(tmp_path / "rhs.bin", rhs)
    out = subprocess.run([exe, "--dist-dump", str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and "DUMPED" in out.stdout, out.stdout + out.stderr
    rel = lambda a, b: np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b)))  # noqa: E731
    for uplo, u in ((orc.LOWER, "L"), (orc.UPPER, "U")):
        F, st = orc.cholesky(spd, uplo, 128)
        assert st == 0
        tri = np.tril if uplo == orc.LOWER else np.triu
        got = _read(tmp_path / f"chol_{u}.bin")
        assert rel(tri(got), tri(F)) <= 1e-11
        other = ~tri(np.ones((n, n), bool))
        assert np.array_equal(got[other], spd[other])
        Xs = orc.cholesky_solve_after(F, rhs, uplo, orc.NORMAL)
        assert rel(_read(tmp_path / f"solveafter_{u}.bin"), Xs) <= 1e-9
        _, Xh, st = orc.hpd_solve(spd, rhs, uplo, nb=128)
        assert rel(_read(tmp_path / f"hpdsolve_{u}.bin"), Xh) <= 1e-9
    Fl, pl, st = orc.lu(ge, 128)
    assert st == 0
    assert np.array_equal(_read(tmp_path / "lu_p.bin", "int32").ravel(), pl)
    assert rel(_read(tmp_path / "lu.bin"), Fl) <= 1e-10
    assert rel(_read(tmp_path / "lusolve.bin"), orc.lu_solve_after(Fl, pl, rhs, orc.NORMAL)) <= 1e-8
    _, Xg, st = orc.gaussian_elimination(ge, rhs, 128)
    assert rel(_read(tmp_path / "gauss.bin"), Xg) <= 1e-8
    for u in ("L", "U"):
        for o in ("N", "T"):
            ref = orc.trsv(u, o, "N", spd, rhs[:, 0])
            assert rel(_read(tmp_path / f"trsv_{u}{o}.bin").ravel(), ref) <= 1e-12
