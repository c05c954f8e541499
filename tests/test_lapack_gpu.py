"""Parity of the GPU LAPACK path with the oracle (the restatement of ATLAS's
recursive getrf/potrf and blocked geqrf): ipiv identical, factors within
rounding, the reference testers' residuals (bin/lutst.c, bin/llttst.c,
bin/qrtst.c, bin/slvtst.c: <= 100), info codes for singular / indefinite
inputs, and lda gaps untouched -- all through the drop-in C ABI."""
import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CM, RM = AB.CblasColMajor, AB.CblasRowMajor


def _getrf_gpu(a, m, n, order=CM):
    ipiv = np.zeros(max(min(m, n), 1), dtype=np.int32)
    info = AB.clapack_dgetrf(order, m, n, a, a.shape[0] if order == CM else a.shape[1], ipiv)
    return ipiv[:min(m, n)], info


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (5, 5), (31, 31), (32, 32), (33, 33), (100, 100),
                                 (257, 257), (600, 600), (700, 300), (300, 700), (1500, 40)])
def test_getrf_vs_oracle_gegen(gpu, orc, m, n):
    lda = m + 3
    a0 = orc.gegen(m, n, lda, m * n + lda)           # the lutst input (random pivots)
    a = a0.copy(order="F")
    ipiv, info = _getrf_gpu(a, m, n)
    ref, rpiv, rinfo = orc.dgetrf(a0.copy(order="F"), m, n)
    assert info == rinfo == 0
    np.testing.assert_array_equal(ipiv, rpiv)
    assert np.max(np.abs(a[:m, :n] - ref[:m, :n])) <= 1e-9
    assert orc.resid_lu(a0[:m, :n].copy(order="F"), a[:m, :n].copy(order="F"), ipiv) <= 100.0
    assert orc.gechkgap(a, m, n) == 0


@pytest.mark.parametrize("n", [64, 513, 1024])
def test_getrf_benchmark_matrix_identity_pivots(gpu, orc, n):
    a0 = orc.lu_matrix(n, 42)
    a = a0.copy(order="F")
    ipiv, info = _getrf_gpu(a, n, n)
    ref, rpiv, _ = orc.dgetrf(a0.copy(order="F"))
    assert info == 0
    np.testing.assert_array_equal(ipiv, rpiv)
    np.testing.assert_array_equal(ipiv, np.arange(n))
    assert orc.resid_lu(a0, a, ipiv) <= 100.0


def test_getrf_singular_info(gpu, orc):
    for col in (0, 6, 39):
        a0 = orc.lu_matrix(40, 5)
        a0[:, col] = 0.0
        a = a0.copy(order="F")
        ipiv, info = _getrf_gpu(a, 40, 40)
        _, rpiv, rinfo = orc.dgetrf(a0.copy(order="F"))
        assert info == rinfo == col + 1
        np.testing.assert_array_equal(ipiv, rpiv)


def test_getrf_row_major(gpu, orc):
    m, n = 60, 45
    a = orc.gegen(m, n, m, 77)[:m, :n]
    R = np.ascontiguousarray(a)              # row-major M x N, lda = N
    ipiv = np.zeros(min(m, n), dtype=np.int32)
    info = AB.clapack_dgetrf(RM, m, n, R, n, ipiv)
    assert info == 0
    # row-major A = L U P (unit U) == column-major factorization of A^T
    ref, rpiv, _ = orc.dgetrf(np.asfortranarray(a.T))
    np.testing.assert_array_equal(ipiv, rpiv)
    np.testing.assert_allclose(R.T, ref, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("trans", [111, 112])
def test_getrs_and_gesv(gpu, orc, trans):
    n, r = 400, 5
    a0 = orc.gegen(n, n, n, 9)
    xt = orc.uniform((n, r), 10)
    b = (a0 if trans == 111 else a0.T) @ xt
    lu = a0.copy(order="F")
    ipiv, info = _getrf_gpu(lu, n, n)
    x = np.array(b, order="F")
    assert AB.clapack_dgetrs(CM, trans, n, r, lu, n, ipiv, x, n) == 0
    A = a0 if trans == 111 else np.asfortranarray(a0.T)
    assert orc.resid_slv(A, x, xt) <= 100.0
    # gesv: A overwritten with its factors, B with the solution
    a = a0.copy(order="F")
    x2 = np.array(a0 @ xt, order="F")
    ip2 = np.zeros(n, dtype=np.int32)
    assert AB.clapack_dgesv(CM, n, r, a, n, ip2, x2, n) == 0
    np.testing.assert_array_equal(ip2, ipiv)
    assert orc.resid_slv(a0, x2, xt) <= 100.0


def test_gesv_row_major(gpu, orc):
    n, r = 200, 3
    a = orc.gegen(n, n, n, 12)
    xt = orc.uniform((n, r), 13)
    rhs = a @ xt                              # each RHS is a column of a @ xt
    Ar = np.ascontiguousarray(a)
    Br = np.asfortranarray(rhs)               # row-major NRHS x N storage == column-major N x NRHS
    ip = np.zeros(n, dtype=np.int32)
    assert AB.clapack_dgesv(RM, n, r, Ar, n, ip, Br, n) == 0
    assert orc.resid_slv(np.asfortranarray(a), Br, xt) <= 100.0


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("n", [1, 4, 5, 63, 64, 65, 200, 700])
def test_potrf_vs_oracle(gpu, orc, uplo, n):
    a0 = orc.spd_matrix(n, 3 + n)
    lda = n + 2
    a = np.zeros((lda, n), order="F")
    a[:n] = a0
    a[n:] = -2560000000.0  # ATL_gegen FILLCONST in the lda gap
    assert AB.clapack_dpotrf(CM, uplo, n, a, lda) == 0
    f = a0.copy(order="F")
    assert orc.dpotrf(uplo, f) == 0
    tri = np.tril if uplo == 122 else np.triu
    assert np.max(np.abs(tri(a[:n]) - tri(f))) <= 1e-11
    assert orc.resid_llt(uplo, a0, a[:n].copy(order="F")) <= 100.0
    assert orc.gechkgap(a, n, n) == 0
    # the other triangle is not touched
    other = np.triu(np.ones((n, n), bool), 1) if uplo == 122 else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(a[:n][other], a0[other])


@pytest.mark.parametrize("bad", [0, 37, 64, 150])
def test_potrf_not_spd_info(gpu, orc, bad):
    n = 200
    a0 = orc.spd_matrix(n, 8)
    a0[bad, bad] = -5.0
    a = a0.copy(order="F")
    info = AB.clapack_dpotrf(CM, 122, n, a, n)
    rinfo = orc.dpotrf(122, a0.copy(order="F"))
    assert info == rinfo == bad + 1


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("r", [13, 32, 40])
def test_potrs_many_rhs(gpu, orc, uplo, r):
    """13 and 32 right-hand sides take the one-launch solves in chunks of 8
    columns, 40 the recursive TRSM: the same solution either way."""
    n = 700
    a0 = orc.spd_matrix(n, 31)
    xt = orc.uniform((n, r), 32)
    f = a0.copy(order="F")
    assert AB.clapack_dpotrf(CM, uplo, n, f, n) == 0
    x = np.array(a0 @ xt, order="F")
    assert AB.clapack_dpotrs(CM, uplo, n, r, f, n, x, n) == 0
    assert orc.resid_slv(a0, x, xt) <= 100.0
    np.testing.assert_allclose(x, xt, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("uplo", [121, 122])
def test_potrs_posv(gpu, orc, uplo):
    n, r = 300, 4
    a0 = orc.spd_matrix(n, 21)
    xt = orc.uniform((n, r), 22)
    a = a0.copy(order="F")
    x = np.array(a0 @ xt, order="F")
    assert AB.clapack_dposv(CM, uplo, n, r, a, n, x, n) == 0
    assert orc.resid_slv(a0, x, xt) <= 100.0
    x2 = np.array(a0 @ xt, order="F")
    assert AB.clapack_dpotrs(CM, uplo, n, r, a, n, x2, n) == 0
    np.testing.assert_allclose(x2, x, rtol=1e-12, atol=1e-12)
    # row-major Upper == column-major Lower on the same buffer
    ar = a0.copy(order="F")
    assert AB.clapack_dpotrf(RM, 121 if uplo == 122 else 122, n, ar, n) == 0
    tri = np.tril if uplo == 122 else np.triu
    np.testing.assert_allclose(tri(ar), tri(a), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("m,n", [(1, 1), (5, 3), (3, 5), (64, 64), (100, 37), (300, 200), (200, 300),
                                 (1000, 130), (700, 700)])
def test_geqrf_vs_oracle(gpu, orc, m, n):
    a0 = orc.normal((m, n), 5 * m + n)
    lda = m + 1
    a = np.full((lda, n), -2560000000.0, order="F")
    a[:m] = a0
    tau = np.zeros(min(m, n))
    assert AB.clapack_dgeqrf(CM, m, n, a, lda, tau) == 0
    qr, rtau = orc.dgeqrf(a0.copy(order="F"))
    k = min(m, n)
    np.testing.assert_allclose(tau, rtau, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(np.triu(a[:m]), np.triu(qr), rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(np.tril(a[:m], -1), np.tril(qr, -1), rtol=1e-8, atol=1e-10)
    assert orc.resid_qr(a0, a[:m].copy(order="F"), tau) <= 100.0
    assert orc.gechkgap(a, m, n) == 0
    assert np.all((tau == 0) | ((tau >= 1) & (tau <= 2)))


def test_geqrf_row_major_is_lq_of_the_view(gpu, orc):
    m, n = 90, 60
    a = orc.normal((m, n), 31)
    R = np.ascontiguousarray(a)               # row-major M x N
    tau = np.zeros(min(m, n))
    assert AB.clapack_dgeqrf(RM, m, n, R, n, tau) == 0
    qr, rtau = orc.dgeqrf(np.asfortranarray(a))
    np.testing.assert_allclose(tau, rtau, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(R, qr, rtol=1e-8, atol=1e-10)


def test_device_api_getrf_potrf(gpu, orc):
    import torch
    n = 256
    a0 = orc.lu_matrix(n, 3)
    A = torch.tensor(a0.T.copy(), device="cuda")   # storage == column-major a0
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert AB.atlb_dgetrf_dev(n, n, A, n, ipiv, info) == 0
    AB.atlb_sync()
    ref, rpiv, _ = orc.dgetrf(a0.copy(order="F"))
    assert int(info.item()) == 0
    np.testing.assert_array_equal(ipiv.cpu().numpy(), rpiv)
    np.testing.assert_allclose(A.cpu().numpy().T, ref, rtol=1e-10, atol=1e-10)


# ------------------------------------------------- pinned to the reference's own LAPACK
import golden_lapack as GL  # noqa: E402


def test_getrf_vs_reference_lapack_golden(gpu):
    """ipiv and info identical to the reference's ATL_getrf (getrfC / getrfR) on
    the testers' sizes, ties in the pivot search, zero columns, row-major and
    1 x n / m x 1 edges; the factors agree to rounding."""
    for i, a, order, lu_ref, ipiv_ref, info_ref in GL.getrf_cases():
        m, n = a.shape
        ipiv = np.zeros(max(min(m, n), 1), dtype=np.int32)
        if order == RM:
            buf = np.ascontiguousarray(a)
            info = AB.clapack_dgetrf(RM, m, n, buf, max(n, 1), ipiv)
            lu = buf
        else:
            lu = a.copy(order="F")
            info = AB.clapack_dgetrf(CM, m, n, lu, max(m, 1), ipiv)
        assert info == info_ref, f"getrf case {i}"
        np.testing.assert_array_equal(ipiv[:min(m, n)], ipiv_ref, err_msg=f"getrf case {i}")
        assert GL.close(lu, lu_ref, 1e-10), f"getrf case {i}"


def test_getrs_vs_reference_lapack_golden(gpu):
    cases = GL.getrf_cases()
    for i, fi, trans, b, x_ref in GL.getrs_cases():
        _, _, _, lu, ipiv, _ = cases[fi]
        n = lu.shape[0]
        x = np.array(b, order="F")
        lu = np.asfortranarray(lu)
        AB.clapack_dgetrs(CM, trans, n, x.shape[1], lu, n, np.ascontiguousarray(ipiv, np.int32), x, n)
        assert GL.close(x, x_ref, 1e-9), f"getrs case {i}"


def test_potrf_potrs_vs_reference_lapack_golden(gpu):
    facs = []
    for i, a, uplo, f_ref, info_ref in GL.potrf_cases():
        n = a.shape[0]
        f = a.copy(order="F")
        info = AB.clapack_dpotrf(CM, uplo, n, f, n)
        facs.append((f, uplo))
        assert info == info_ref, f"potrf case {i}"
        k = n if info == 0 else info - 1
        assert GL.close(GL.tri(f, uplo)[:k, :k], f_ref[:k, :k], 1e-11), f"potrf case {i}"
    for i, fi, b, x_ref in GL.potrs_cases():
        f, uplo = facs[fi]
        n = f.shape[0]
        x = np.array(b, order="F")
        AB.clapack_dpotrs(CM, uplo, n, x.shape[1], f, n, x, n)
        assert GL.close(x, x_ref, 1e-9), f"potrs case {i}"


def test_geqrf_vs_reference_lapack_golden(gpu):
    """R, the Householder vectors and tau of the reference's ATL_geqrf
    (ATLAS's larfg sign and tau conventions)."""
    for i, a, qr_ref, tau_ref, info_ref in GL.geqrf_cases():
        m, n = a.shape
        qr = a.copy(order="F")
        tau = np.zeros(max(min(m, n), 1))
        info = AB.clapack_dgeqrf(CM, m, n, qr, max(m, 1), tau)
        assert info == info_ref == 0, f"geqrf case {i}"
        assert GL.close(qr, qr_ref, 1e-10), f"geqrf case {i}"
        assert GL.close(tau[:min(m, n)], tau_ref, 1e-10), f"geqrf case {i}"


@pytest.mark.parametrize("m,n", [(300, 900), (900, 300), (257, 385), (129, 129), (640, 129)])
def test_geqrf_lookahead_shapes_vs_oracle(gpu, orc, m, n):
    """Wide, tall and ragged shapes through the look-ahead driver: the last
    panel narrower than the others, a wide matrix whose columns beyond
    min(m, n) get only the block reflectors, a single extra column."""
    a0 = orc.normal((m, n), 3 * m + n)
    a = a0.copy(order="F")
    tau = np.zeros(min(m, n))
    assert AB.clapack_dgeqrf(CM, m, n, a, m, tau) == 0
    qr, rtau = orc.dgeqrf(a0.copy(order="F"))
    np.testing.assert_allclose(tau, rtau, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(np.triu(a), np.triu(qr), rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(np.tril(a, -1), np.tril(qr, -1), rtol=1e-8, atol=1e-10)
    assert orc.resid_qr(a0, a.copy(order="F"), tau) <= 100.0


@pytest.mark.parametrize("n", [129, 300, 513])
@pytest.mark.parametrize("uplo", [121, 122])
def test_potrf_lookahead_sizes_vs_oracle(gpu, orc, n, uplo):
    """Orders just past one, two and four 128-column blocks through the
    Cholesky look-ahead (the last block narrow), both triangles."""
    a0 = orc.spd_matrix(n, 7 * n)
    a = a0.copy(order="F")
    assert AB.clapack_dpotrf(CM, uplo, n, a, n) == 0
    f = a0.copy(order="F")
    assert orc.dpotrf(uplo, f) == 0
    tri = np.triu if uplo == 121 else np.tril
    np.testing.assert_allclose(tri(a), tri(f), rtol=1e-10, atol=1e-11)


@pytest.mark.parametrize("nb", [64, 256])
@pytest.mark.parametrize("la", [0, 1])
def test_geqrf_panel_widths_vs_oracle(gpu, orc, nb, la):
    """qr_nb = 256 factors each panel as two 128-column halves (the left
    half's block reflector applied to the right half in between, T built
    from the two halves' T); with and without look-ahead the result matches
    the oracle as with the default width, and so does Q applied by dormqr."""
    m, n = 1100, 700
    a0 = orc.normal((m, n), 97)
    try:
        assert AB.atlb_tune_set("qr_nb", nb) == nb
        assert AB.atlb_tune_set("lookahead", la) == la
        a = a0.copy(order="F")
        tau = np.zeros(n)
        assert AB.clapack_dgeqrf(CM, m, n, a, m, tau) == 0
        qr, rtau = orc.dgeqrf(a0.copy(order="F"))
        np.testing.assert_allclose(tau, rtau, rtol=1e-9, atol=1e-11)
        np.testing.assert_allclose(np.triu(a), np.triu(qr), rtol=1e-9, atol=1e-10)
        np.testing.assert_allclose(np.tril(a, -1), np.tril(qr, -1), rtol=1e-8, atol=1e-10)
        assert orc.resid_qr(a0, a.copy(order="F"), tau) <= 100.0
        # Q^T A = R through the blocked apply at the same width
        c = a0.copy(order="F")
        assert AB.ATL_dormqr(AB.CblasLeft, AB.CblasTrans, m, n, n, a, m, tau, c, m, None, 0) == 0
        r = np.triu(a)[:n]
        np.testing.assert_allclose(c[:n], r, rtol=1e-9, atol=1e-9 * np.abs(r).max())
        assert np.abs(c[n:]).max() <= 1e-9 * np.abs(r).max()
    finally:
        AB.atlb_tune_set("qr_nb", 128)
        AB.atlb_tune_set("lookahead", 1)
