"""The oracle pinned to the reference itself: the C restatement (liboracle.so,
oracle/oref_impl.h) against the reference's own code compiled from its sources
(oracle/_ref/libelemref.so, oracle/refbuild/) on the same seeded inputs, and
against the golden vectors that the reference produced
(tests/golden/make_golden.py -> tests/golden/ref_golden.npz).

Tolerances: pivot vectors, row interchanges and every integer result
identical; floating-point results to rounding (the reference's level-3 flops
run in OpenBLAS, the restatement in netlib loop order): 1e-12 relative for
factors of well-conditioned inputs, 1e-10 for solves and inverses."""
import os

import numpy as np
import pytest

from elemental_b200 import inputs
from oracle import pyoracle as orc
from oracle import ref

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ref_golden.npz")

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (needs the reference sources)")


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


# ------------------------------------------------------- golden vectors --

def test_golden_vectors_pin_the_restatement():
    g = np.load(GOLDEN)
    for key in [k for k in g.files if k.startswith("chol_in_")]:
        tag = key[len("chol_in_"):]
        n, uplo, nb = (int(x) for x in tag.split("_"))
        F, st = orc.cholesky(g[key], uplo, nb)
        assert st == 0
        tri = np.tril if uplo == orc.LOWER else np.triu
        assert rel(tri(F), tri(g["chol_out_" + tag])) <= 1e-12
    for key in [k for k in g.files if k.startswith("lu_in_")]:
        tag = key[len("lu_in_"):]
        F, p, st = orc.lu(g[key], 128)
        assert st == 0
        assert np.array_equal(p, g["lu_piv_" + tag])
        assert rel(F, g["lu_out_" + tag]) <= 1e-12
        X = orc.lu_solve_after(F, p, g["lu_rhs_" + tag], orc.NORMAL)
        assert rel(X, g["lu_x_" + tag]) <= 1e-10
    for key in [k for k in g.files if k.startswith("lurect_in_")]:
        tag = key[len("lurect_in_"):]
        F, p, st = orc.lu(g[key], 128)
        assert st == 0 and np.array_equal(p, g["lurect_piv_" + tag]) and rel(F, g["lurect_out_" + tag]) <= 1e-12
    _, X, st = orc.hpd_solve(g["hpd_A"], g["hpd_B"], orc.LOWER, nb=128)
    assert st == 0 and rel(X, g["hpd_X"]) <= 1e-10
    _, X, st = orc.gaussian_elimination(g["ge_A"], g["ge_B"], 128)
    assert st == 0 and rel(X, g["ge_X"]) <= 1e-10
    assert np.array_equal(orc.apply_row_pivots(g["swap_B"], g["swap_p"]), g["swap_out"])
    assert np.array_equal(orc.apply_row_pivots(g["swap_B"], g["swap_p"], True), g["swap_out_inv"])


# ------------------------------------- the restatement against the reference --

@needs_ref
@pytest.mark.parametrize("n", [1, 7, 127, 128, 129, 300, 1000])
@pytest.mark.parametrize("uplo", [orc.LOWER, orc.UPPER])
def test_cholesky_matches_reference(n, uplo):
    A = inputs.spd_ggt(n, 10 + n)
    for nb in (32, 96, 128):
        R, st_r = ref.cholesky(A, uplo, nb)
        O, st_o = orc.cholesky(A, uplo, nb)
        assert st_r == st_o == 0
        assert np.array_equal(R, O) or rel(R, O) <= 1e-12
        other = ~(np.tril if uplo == orc.LOWER else np.triu)(np.ones((n, n), bool))
        assert np.array_equal(R[other], A[other]) and np.array_equal(O[other], A[other])


@needs_ref
def test_cholesky_dist_1x1_matches_reference_sequential():
    A = inputs.spd_ggt(400, 5)
    for uplo in (orc.LOWER, orc.UPPER):
        R, _ = ref.cholesky(A, uplo, 96)
        D, st = ref.cholesky(A, uplo, 96, dist=True)
        O, _ = orc.cholesky(A, uplo, 96)
        tri = np.tril if uplo == orc.LOWER else np.triu
        assert st == 0 and rel(tri(D), tri(R)) <= 1e-12 and rel(tri(O), tri(D)) <= 1e-12


@needs_ref
def test_not_hpd_and_singular_statuses_match_reference():
    A = inputs.spd_ggt(300, 3)
    A[200, 200] = -5.0
    assert ref.cholesky(A, orc.LOWER)[1] == 1
    assert orc.cholesky(A, orc.LOWER)[1] == 201  # the restatement also names the column
    S = inputs.uniform(300, 300, 77)
    S[:, 150] = 0.0
    assert ref.lu(S)[2] == 2
    assert orc.lu(S, 128)[2] == 151


@needs_ref
@pytest.mark.parametrize("shape", [(1, 1), (7, 7), (129, 129), (300, 300), (1000, 1000), (500, 300), (300, 500),
                                   (1000, 129)])
def test_lu_pivots_index_for_index(shape):
    m, n = shape
    A = inputs.uniform(m, n, m * 7 + n)
    for nb in (32, 128):
        R, pr, st_r = ref.lu(A, nb)
        O, po, st_o = orc.lu(A, nb)
        assert st_r == st_o == 0
        assert np.array_equal(pr, po), np.nonzero(pr != po)[0][:10]
        assert rel(O, R) <= 1e-12
    D, pd, st = ref.lu(A, 128, dist=True)
    assert st == 0 and np.array_equal(pd, po) and rel(D, R) <= 1e-12


@needs_ref
def test_lu_nopiv_matches_reference():
    A = inputs.uniform(500, 500, 8) + 500 * np.eye(500)
    R, st = ref.lu_nopiv(A, 128)
    O, st2 = orc.lu_nopiv(A, 128)
    assert st == st2 == 0 and rel(O, R) <= 1e-12


@needs_ref
@pytest.mark.parametrize("orient", [orc.NORMAL, orc.TRANSPOSE])
@pytest.mark.parametrize("nrhs", [1, 7])
def test_solves_match_reference(orient, nrhs):
    n = 401
    A = inputs.uniform(n, n, 31)
    B = inputs.normal(n, nrhs, 32)
    F, p, _ = ref.lu(A, 128)
    assert rel(orc.lu_solve_after(F, p, B, orient), ref.lu_solve_after(F, p, B, orient)) <= 1e-10
    assert rel(ref.lu_solve_after(F, p, B, orient, dist=True), ref.lu_solve_after(F, p, B, orient)) <= 1e-12
    H = inputs.spd_ggt(n, 33)
    for uplo in (orc.LOWER, orc.UPPER):
        _, Xr, st = ref.hpd_solve(H, B, uplo, orient)
        _, Xo, st2 = orc.hpd_solve(H, B, uplo, orient)
        _, Xd, st3 = ref.hpd_solve(H, B, uplo, orient, dist=True)
        assert st == st2 == st3 == 0 and rel(Xo, Xr) <= 1e-10 and rel(Xd, Xr) <= 1e-10
        Fh, _ = ref.cholesky(H, uplo)
        assert rel(orc.cholesky_solve_after(Fh, B, uplo, orient), ref.cholesky_solve_after(Fh, B, uplo, orient)) <= 1e-10


@needs_ref
def test_gaussian_elimination_matches_reference_distributed_form():
    # the restatement follows the distributed RowEchelon (the reference's
    # sequential RowEchelon crashes; see oracle/refbuild/glue.cpp)
    n = 333
    A = inputs.uniform(n, n, 41)
    B = inputs.normal(n, 5, 42)
    Fr, Xr, st = ref.gaussian_elimination(A, B)
    Fo, Xo, st2 = orc.gaussian_elimination(A, B, 128)
    assert st == st2 == 0
    assert rel(np.triu(Fo), np.triu(Fr)) <= 1e-12 and rel(Xo, Xr) <= 1e-10


@needs_ref
@pytest.mark.parametrize("inverse", [False, True])
def test_apply_row_pivots_bit_exact(inverse):
    n = 513
    r = inputs.rng(5)
    p = np.array([i + r.integers(0, n - i) for i in range(n)], dtype=np.int32)
    B = inputs.normal(n, 7, 6)
    assert np.array_equal(orc.apply_row_pivots(B, p, inverse), ref.apply_row_pivots(B, p, inverse))


@needs_ref
def test_blas_wrappers_match_reference():
    r = inputs.rng(9)
    n, k = 150, 40
    A = np.asfortranarray(r.uniform(-1, 1, (n, n)) / np.sqrt(n) + 2 * np.eye(n))
    B = np.asfortranarray(r.standard_normal((n, k)))
    names = {orc.LOWER: "L", orc.UPPER: "U"}
    for uplo in (orc.LOWER, orc.UPPER):
        for orient in (orc.NORMAL, orc.TRANSPOSE):
            for diag in (0, 1):
                o = orc.trsm("L", names[uplo], "NT"[orient], "NU"[diag], 0.5, A, B)
                assert rel(o, ref.trsm(0, uplo, orient, diag, 0.5, A, B)) <= 1e-12
                o = orc.trsm("R", names[uplo], "NT"[orient], "NU"[diag], 0.5, A, B.T.copy(order="F"))
                assert rel(o, ref.trsm(1, uplo, orient, diag, 0.5, A, B.T.copy(order="F"))) <= 1e-12
                assert rel(orc.trsv(names[uplo], "NT"[orient], "NU"[diag], A, B[:, 0]),
                           ref.trsv(uplo, orient, diag, A, B[:, 0])) <= 1e-12
    C = np.asfortranarray(r.standard_normal((n, n)))
    assert rel(orc.gemm("N", "T", -1.0, B, B, 1.0, C), ref.gemm(0, 1, -1.0, B, B, 1.0, C)) <= 1e-12
    for uplo in (orc.LOWER, orc.UPPER):
        o = orc.syrk(names[uplo], "N", -1.0, B, 1.0, C)
        R = ref.herk(uplo, orc.NORMAL, -1.0, B, 1.0, C)
        tri = np.tril if uplo == orc.LOWER else np.triu
        assert rel(tri(o), tri(R)) <= 1e-12
        assert np.array_equal(R[~tri(np.ones((n, n), bool))], C[~tri(np.ones((n, n), bool))])


@needs_ref
def test_next_rows_match_reference():
    n = 260
    H = inputs.spd_ggt(n, 50)
    G = inputs.uniform(n, n, 51) + 4 * np.eye(n)
    assert rel(orc.inverse(G, 128)[0], ref.inverse(G, 128)[0]) <= 1e-10
    for uplo in (orc.LOWER, orc.UPPER):
        tri = np.tril if uplo == orc.LOWER else np.triu
        assert rel(tri(orc.hpd_inverse(H, uplo, 128)[0]), tri(ref.hpd_inverse(H, uplo, 128)[0])) <= 1e-10
        for unit in (False, True):
            T = tri(G)
            assert rel(tri(orc.triangular_inverse(T, uplo, unit)), tri(ref.triangular_inverse(T, uplo, unit))) <= 1e-10
    Lo, do, _ = orc.ldl(H)
    Lr, dr, st = ref.ldl(H)
    assert st == 0 and rel(do, dr) <= 1e-12 and rel(np.tril(Lo, -1), np.tril(Lr, -1)) <= 1e-12
    (rho_o, kap_o), (rho_r, kap_r) = orc.safe_determinant(G)[:2], ref.safe_determinant(G)
    assert rho_o == rho_r and abs(kap_o - kap_r) <= 1e-12 * abs(kap_r)
    (rho_o, kap_o), (rho_r, kap_r) = orc.safe_hpd_determinant(H)[:2], ref.safe_determinant(H, hpd=True)
    assert rho_o == rho_r and abs(kap_o - kap_r) <= 1e-12 * abs(kap_r)


@needs_ref
@pytest.mark.parametrize("uplo", [orc.LOWER, orc.UPPER])
def test_reverse_cholesky_matches_reference_within_one_block(uplo):
    # n <= Blocksize(): the reference runs ReverseLVar3Unb / ReverseUVar3Unb
    # alone (Cholesky/LVar3.hpp:50-79) and the restatement matches it exactly
    H = inputs.spd_ggt(120, 52)
    tri = np.tril if uplo == orc.LOWER else np.triu
    R, st = ref.reverse_cholesky(H, uplo, 128)
    assert st == 0
    assert np.array_equal(tri(orc.reverse_cholesky(H, uplo)[0]), tri(R))


@needs_ref
@pytest.mark.parametrize("uplo", [orc.LOWER, orc.UPPER])
def test_reverse_cholesky_reference_blocked_form_is_not_a_factorization(uplo):
    # Recorded deviation.  The reference's blocked ReverseLVar3
    # (Cholesky/LVar3.hpp:125-165) solves A10 := inv(L11) A10 with
    # Trsm(LEFT, LOWER, NORMAL), but A = L^T L gives A10 = L11^T L10, which
    # needs the adjoint; ReverseUVar3 (Cholesky/UVar3.hpp) mirrors it.  For
    # n > Blocksize() its result does not factor A.  The restatement and the GPU
    # path return the factor that ReverseLVar3Unb defines (A = L^T L, resp.
    # A = U U^T), which is what the reference returns for n <= Blocksize().
    H = inputs.spd_ggt(260, 50)
    tri = np.tril if uplo == orc.LOWER else np.triu
    R = tri(ref.reverse_cholesky(H, uplo, 32)[0])
    O = tri(orc.reverse_cholesky(H, uplo)[0])
    res = (lambda T: T.T @ T) if uplo == orc.LOWER else (lambda T: T @ T.T)
    assert rel(res(R), H) > 1e-3
    assert rel(res(O), H) <= 1e-14
