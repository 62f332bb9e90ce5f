"""Generate tests/golden/ref_golden.npz from the reference's own code
(oracle/_ref/libelemref.so, built from the reference sources by
oracle/refbuild/Makefile).  Small seeded cases: Cholesky (both triangles,
block sizes 32/96/128), LU with partial pivoting + lu::SolveAfter (square and
rectangular), HPDSolve, GaussianElimination (1 x 1 Grid form) and
ApplyRowPivots / ApplyInverseRowPivots.  The fixture travels with the tests,
so the pin holds where the reference sources are absent.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from elemental_b200 import inputs  # noqa: E402
from oracle import ref  # noqa: E402


def main():
    ref.build()
    out = {}
    for n, uplo, nb in ((1, 0, 128), (7, 1, 32), (130, 0, 128), (97, 1, 32)):
        A = inputs.spd_ggt(n, 900 + n)
        F, st = ref.cholesky(A, uplo, nb)
        assert st == 0
        tag = f"{n}_{uplo}_{nb}"
        out["chol_in_" + tag], out["chol_out_" + tag] = A, F
    for m, n in ((1, 1), (40, 40), (131, 131), (120, 70), (70, 120)):
        A = inputs.uniform(m, n, 1000 + m + 3 * n)
        F, p, st = ref.lu(A, 128)
        assert st == 0
        tag = f"{m}_{n}"
        out["lu_in_" + tag], out["lu_out_" + tag], out["lu_piv_" + tag] = A, F, p
        if m == n:
            B = inputs.normal(n, 3, 2000 + n)
            out["lu_rhs_" + tag], out["lu_x_" + tag] = B, ref.lu_solve_after(F, p, B)
    A = inputs.spd_ggt(100, 31)
    B = inputs.normal(100, 4, 32)
    out["hpd_A"], out["hpd_B"] = A, B
    out["hpd_X"] = ref.hpd_solve(A, B, 0)[1]
    A = inputs.uniform(90, 90, 41)
    B = inputs.normal(90, 2, 42)
    out["ge_A"], out["ge_B"] = A, B
    out["ge_X"] = ref.gaussian_elimination(A, B)[1]
    r = inputs.rng(5)
    p = np.array([i + r.integers(0, 97 - i) for i in range(97)], dtype=np.int32)
    B = inputs.normal(97, 3, 6)
    out["swap_B"], out["swap_p"] = B, p
    out["swap_out"], out["swap_out_inv"] = ref.apply_row_pivots(B, p), ref.apply_row_pivots(B, p, True)
    # keep only the square LU cases' solve keys consistent
    for k in [k for k in out if k.startswith("lu_in_")]:
        tag = k[len("lu_in_"):]
        if "lu_rhs_" + tag not in out:
            m, n = (int(x) for x in tag.split("_"))
            del out["lu_in_" + tag]
            out["lurect_in_" + tag], out["lurect_out_" + tag], out["lurect_piv_" + tag] = (
                inputs.uniform(m, n, 1000 + m + 3 * n), out.pop("lu_out_" + tag), out.pop("lu_piv_" + tag))
    out["blas_config"] = np.array(ref.blas_config())
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_golden.npz"), **out)


if __name__ == "__main__":
    main()
