"""Pins the CPU oracle (the checker of the GPU library) before it is trusted:
its generator against the LCG it restates, its BLAS against the reference's
own C reference BLAS outputs (tests/golden/ref_blas.npz, generated from
oracle/_ref by tests/golden/make_golden.py), and its LAPACK against the
reference testers' residual criteria and LAPACK's conventions (scipy)."""
import os

import numpy as np
import pytest
import scipy.linalg as sla

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_blas.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("seed", [1, 7, 1234, 65535])
def test_lcg_is_the_ansi_c_lcg(orc, seed):
    # ATL_rand (src/testing/ATL_rand.c) = x' = (1103515245 x + 12345) mod 2^31
    lib = orc.orc()
    lib.orc_srand(seed)
    x = (1103515245 * seed + 12345) % (1 << 31)
    for _ in range(2000):
        assert lib.orc_rand() == x
        x = (1103515245 * x + 12345) % (1 << 31)


def test_gegen_range_and_gap(orc):
    a = orc.gegen(37, 11, 41, 99)
    v = a[:37, :11]
    assert np.all(v > -0.5) and np.all(v <= 0.5)
    assert orc.gechkgap(a, 37, 11) == 0
    a[38, 3] = 0.0
    assert orc.gechkgap(a, 37, 11) == 1


def _close(x, y, scale):
    return np.max(np.abs(x - y)) <= 1e-13 * max(1.0, scale)


def test_oracle_gemm_matches_reference_blas(orc, gold):
    for i in range(int(gold["counts"][0])):
        m, n, k, ta, tb, alpha, beta = gold[f"gemm{i}"]
        m, n, k, ta, tb = int(m), int(n), int(k), int(ta), int(tb)
        a, b = gold[f"gemm{i}_A"], gold[f"gemm{i}_B"]
        c = np.array(gold[f"gemm{i}_C0"], order="F")
        orc.dgemm(ta, tb, m, n, k, alpha, a, b, beta, c)
        ref = gold[f"gemm{i}_C"]
        assert _close(c[:m, :n], ref[:m, :n], k), f"gemm case {i}"
        assert orc.gechkgap(c, m, n) == 0


def test_oracle_trsm_trmm_match_reference_blas(orc, gold):
    for i in range(int(gold["counts"][1])):
        m, n, side, uplo, ta, diag, alpha = gold[f"trsm{i}"]
        m, n, side, uplo, ta, diag = map(int, (m, n, side, uplo, ta, diag))
        a = gold[f"trsm{i}_A"]
        b = np.array(gold[f"trsm{i}_B0"], order="F")
        orc.dtrsm(side, uplo, ta, diag, m, n, alpha, a, b)
        assert _close(b[:m, :n], gold[f"trsm{i}_X"][:m, :n], max(m, n)), f"trsm case {i}"
        bm = np.array(gold[f"trsm{i}_B0"], order="F")
        orc.dtrmm(side, uplo, ta, diag, m, n, alpha, a, bm)
        assert _close(bm[:m, :n], gold[f"trsm{i}_TB"][:m, :n], max(m, n)), f"trmm case {i}"


def test_oracle_syrk_matches_reference_blas(orc, gold):
    for i in range(int(gold["counts"][2])):
        n, k, uplo, tr, alpha, beta = gold[f"syrk{i}"]
        n, k, uplo, tr = map(int, (n, k, uplo, tr))
        a = gold[f"syrk{i}_A"]
        c = np.array(gold[f"syrk{i}_C0"], order="F")
        orc.dsyrk(uplo, tr, n, k, alpha, a, beta, c)
        ref = gold[f"syrk{i}_C"]
        assert _close(c[:n, :n], ref[:n, :n], k), f"syrk case {i}"


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_oracle_gemm_matches_live_reference(orc):
    R = O.ref()
    for ta in (O.NoTrans, O.Trans):
        for tb in (O.NoTrans, O.Trans):
            m, n, k = 57, 43, 61
            a = O.uniform((61, 61), 1)
            b = O.uniform((61, 61), 2)
            c1 = O.uniform((m, n), 3)
            c2 = c1.copy(order="F")
            R.ATL_drefgemm(ta, tb, m, n, k, 0.5, O.P(a), 61, O.P(b), 61, 2.0, O.P(c1), m)
            O.dgemm(ta, tb, m, n, k, 0.5, a, b, 2.0, c2)
            assert _close(c1, c2, k)


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (7, 7), (50, 50), (130, 130), (90, 40), (40, 90)])
def test_oracle_getrf_matches_lapack(orc, m, n):
    a0 = orc.gegen(m, n, m, m * n + m)[:m, :n].copy(order="F")
    lu, ipiv, info = orc.dgetrf(a0.copy(order="F"))
    assert info == 0
    plu, ppiv = sla.lu_factor(a0, check_finite=False)
    k = min(m, n)
    np.testing.assert_array_equal(ipiv, ppiv[:k])
    np.testing.assert_allclose(lu, plu, rtol=1e-10, atol=1e-12)
    assert orc.resid_lu(a0, lu, ipiv) <= 100.0


def test_oracle_getrf_zero_pivot_info(orc):
    a = orc.lu_matrix(20, 5)
    a[:, 6] = 0.0
    lu, ipiv, info = orc.dgetrf(a.copy(order="F"))
    assert info == 7


@pytest.mark.parametrize("uplo", [O.Lower, O.Upper])
@pytest.mark.parametrize("n", [1, 3, 5, 17, 100])
def test_oracle_potrf_matches_numpy(orc, uplo, n):
    a0 = orc.spd_matrix(n, 11 + n)
    f = a0.copy(order="F")
    assert orc.dpotrf(uplo, f) == 0
    L = np.linalg.cholesky(a0)
    if uplo == O.Lower:
        np.testing.assert_allclose(np.tril(f), L, rtol=1e-12, atol=1e-13)
    else:
        np.testing.assert_allclose(np.triu(f), L.T, rtol=1e-12, atol=1e-13)
    assert orc.resid_llt(uplo, a0, f) <= 100.0


def test_oracle_potrf_not_spd_info(orc):
    a = orc.spd_matrix(12, 3)
    a[8, 8] = -1.0
    assert orc.dpotrf(O.Lower, a.copy(order="F")) == 9


@pytest.mark.parametrize("m,n,nb", [(1, 1, 32), (5, 3, 2), (60, 40, 8), (40, 60, 8), (200, 100, 32), (97, 97, 16)])
def test_oracle_geqrf_matches_lapack(orc, m, n, nb):
    a0 = orc.normal((m, n), m + 31 * n)
    qr, tau = orc.dgeqrf(a0.copy(order="F"), nb)
    (pqr, ptau), _r = sla.qr(a0, mode="raw")
    k = min(m, n)
    np.testing.assert_allclose(np.triu(qr), np.triu(pqr), rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(tau, ptau[:k], rtol=1e-9, atol=1e-12)
    assert np.all((tau == 0) | ((tau >= 1) & (tau <= 2)))
    assert orc.resid_qr(a0, qr, tau) <= 100.0


def test_oracle_getrs_potrs_solve(orc):
    n, r = 60, 3
    a0 = orc.lu_matrix(n, 8)
    xt = orc.uniform((n, r), 9)
    b = a0 @ xt
    lu, ipiv, _ = orc.dgetrf(a0.copy(order="F"))
    x = orc.dgetrs(O.NoTrans, lu, ipiv, np.array(b, order="F"))
    assert orc.resid_slv(a0, x, xt) <= 100.0
    bt = a0.T @ xt
    x = orc.dgetrs(O.Trans, lu, ipiv, np.array(bt, order="F"))
    assert orc.resid_slv(a0.T.copy(order="F"), x, xt) <= 100.0
    s0 = orc.spd_matrix(n, 4)
    f = s0.copy(order="F")
    orc.dpotrf(O.Upper, f)
    x = orc.dpotrs(O.Upper, f, np.array(s0 @ xt, order="F"))
    assert orc.resid_slv(s0, x, xt) <= 100.0


def test_residuals_detect_errors(orc):
    a0 = orc.lu_matrix(40, 2)
    lu, ipiv, _ = orc.dgetrf(a0.copy(order="F"))
    assert orc.resid_lu(a0, lu, ipiv) < 10
    bad = lu.copy(order="F")
    bad[30, 31] += 1e-6
    assert orc.resid_lu(a0, bad, ipiv) > 100


def test_ddgemm_is_more_accurate_than_fp64(orc):
    a = orc.uniform((30, 200), 5)
    b = orc.uniform((200, 20), 6)
    hi, lo = orc.ddgemm(a, b)
    c = a @ b
    err = orc.normwise_err_dd(np.asfortranarray(c), hi, lo)
    assert 0 < err < 1e-14
    assert orc.normwise_err_dd(hi, hi, lo) < 1e-15  # only the low word remains
