"""The rest of the level-3 BLAS and the inverse / least-squares LAPACK routines
of the C interface (cblas_dsymm / dsyr2k / zgemm, clapack_dgetri / dtrtri /
dlauum / dpotri / dgels / dgelqf, ATL_dormqr) and the Fortran 77 calling
convention, through the C ABI with host arrays, against FP64 numpy (and the
oracle's QR for gelqf).  Both storage orders where the interface has them."""
import ctypes

import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CM, RM = AB.CblasColMajor, AB.CblasRowMajor
L_, R_, U_, LO = AB.CblasLeft, AB.CblasRight, AB.CblasUpper, AB.CblasLower
NT, TR, CT = AB.CblasNoTrans, AB.CblasTrans, AB.CblasConjTrans


def _rng(s):
    return np.random.default_rng(s)


def _store(a, order):
    """(buffer, ld) holding the logical matrix a in the given storage order."""
    if order == CM:
        return np.array(a, order="F", copy=True), max(1, a.shape[0])
    return np.array(a, order="C", copy=True), max(1, a.shape[1])


def _logical(buf, order):
    return np.array(buf) if order == RM else np.array(buf, order="F")


def _rel(x, y):
    return np.max(np.abs(x - y)) / max(1e-300, np.max(np.abs(y)))


@pytest.mark.parametrize("order", [CM, RM])
@pytest.mark.parametrize("side", [L_, R_])
@pytest.mark.parametrize("uplo", [U_, LO])
def test_dsymm(gpu, order, side, uplo):
    m, n = 130, 77
    r = _rng(1)
    na = m if side == L_ else n
    s = r.uniform(-1, 1, (na, na))
    sym = np.triu(s) + np.triu(s, 1).T if uplo == U_ else np.tril(s) + np.tril(s, -1).T
    a = s.copy()  # only the `uplo` triangle is referenced
    b = r.uniform(-1, 1, (m, n))
    c = r.uniform(-1, 1, (m, n))
    ref = 0.7 * (sym @ b if side == L_ else b @ sym) - 1.3 * c
    A, lda = _store(a, order)
    B, ldb = _store(b, order)
    C, ldc = _store(c, order)
    AB.cblas_dsymm(order, side, uplo, m, n, 0.7, A, lda, B, ldb, -1.3, C, ldc)
    assert _rel(_logical(C, order), ref) < 1e-13


@pytest.mark.parametrize("order", [CM, RM])
@pytest.mark.parametrize("trans", [NT, TR])
@pytest.mark.parametrize("uplo", [U_, LO])
def test_dsyr2k(gpu, order, trans, uplo):
    n, k = 150, 61
    r = _rng(2)
    shape = (n, k) if trans == NT else (k, n)
    a = r.uniform(-1, 1, shape)
    b = r.uniform(-1, 1, shape)
    c0 = r.uniform(-1, 1, (n, n))
    full = 0.5 * (a @ b.T + b @ a.T) if trans == NT else 0.5 * (a.T @ b + b.T @ a)
    full += 2.0 * c0
    A, lda = _store(a, order)
    B, ldb = _store(b, order)
    C, ldc = _store(c0, order)
    AB.cblas_dsyr2k(order, uplo, trans, n, k, 0.5, A, lda, B, ldb, 2.0, C, ldc)
    out = _logical(C, order)
    tri = np.triu if uplo == U_ else np.tril
    other = np.tril if uplo == U_ else np.triu
    assert _rel(tri(out), tri(full)) < 1e-13
    off = -1 if uplo == U_ else 1
    np.testing.assert_array_equal(other(out, off), other(c0, off))  # the other triangle is untouched


@pytest.mark.parametrize("order", [CM, RM])
@pytest.mark.parametrize("ta,tb", [(NT, NT), (TR, NT), (NT, CT), (CT, TR), (CT, CT)])
def test_zgemm(gpu, order, ta, tb):
    m, n, k = 90, 70, 55
    r = _rng(3)
    opa = lambda x, t: x if t == NT else (x.T if t == TR else x.conj().T)
    a = r.uniform(-1, 1, (m, k) if ta == NT else (k, m)) + 1j * r.uniform(-1, 1, (m, k) if ta == NT else (k, m))
    b = r.uniform(-1, 1, (k, n) if tb == NT else (n, k)) + 1j * r.uniform(-1, 1, (k, n) if tb == NT else (n, k))
    c = r.uniform(-1, 1, (m, n)) + 1j * r.uniform(-1, 1, (m, n))
    alpha, beta = 0.5 - 0.25j, 1.5 + 0.5j
    ref = alpha * opa(a, ta) @ opa(b, tb) + beta * c
    A, lda = _store(a, order)
    B, ldb = _store(b, order)
    C, ldc = _store(c, order)
    al = np.array([alpha], np.complex128)
    be = np.array([beta], np.complex128)
    AB.cblas_zgemm(order, ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc)
    assert _rel(_logical(C, order), ref) < 1e-13


@pytest.mark.parametrize("order", [CM, RM])
def test_dgetri(gpu, order):
    n = 300
    a = O.gegen(n, n, n, 7)[:n, :n]
    A, lda = _store(a, order)
    ipiv = np.zeros(n, np.int32)
    assert AB.clapack_dgetrf(order, n, n, A, lda, ipiv) == 0
    assert AB.clapack_dgetri(order, n, A, lda, ipiv) == 0
    inv = _logical(A, order)
    assert np.max(np.abs(inv @ a - np.eye(n))) < 1e-10


def test_dgetri_singular(gpu):
    n = 50
    a = O.gegen(n, n, n, 8)[:n, :n].copy(order="F")
    a[:, 10] = 0.0
    ipiv = np.zeros(n, np.int32)
    assert AB.clapack_dgetrf(CM, n, n, a, n, ipiv) == 11
    assert AB.clapack_dgetri(CM, n, a, n, ipiv) > 0


@pytest.mark.parametrize("order", [CM, RM])
@pytest.mark.parametrize("uplo", [U_, LO])
@pytest.mark.parametrize("diag", [AB.CblasNonUnit, AB.CblasUnit])
def test_dtrtri(gpu, order, uplo, diag):
    n = 200
    r = _rng(4)
    a = r.uniform(-1, 1, (n, n)) / n + 2 * np.eye(n)
    t = np.triu(a) if uplo == U_ else np.tril(a)
    if diag == AB.CblasUnit:
        t = t - np.diag(np.diag(t)) + np.eye(n)
    A, lda = _store(a, order)
    assert AB.clapack_dtrtri(order, uplo, diag, n, A, lda) == 0
    out = _logical(A, order)
    tri = np.triu if uplo == U_ else np.tril
    inv = tri(out)
    if diag == AB.CblasUnit:
        np.testing.assert_array_equal(np.diag(out), np.diag(a))  # the diagonal is not referenced
        inv = inv - np.diag(np.diag(inv)) + np.eye(n)
    assert np.max(np.abs(inv @ t - np.eye(n))) < 1e-12
    other = np.tril if uplo == U_ else np.triu
    off = -1 if uplo == U_ else 1
    np.testing.assert_array_equal(other(out, off), other(a, off))


@pytest.mark.parametrize("order", [CM, RM])
@pytest.mark.parametrize("uplo", [U_, LO])
def test_dlauum_and_dpotri(gpu, order, uplo):
    n = 180
    spd = O.spd_matrix(n, 5)
    A, lda = _store(spd, order)
    assert AB.clapack_dpotrf(order, uplo, n, A, lda) == 0
    f = _logical(A, order)
    t = np.triu(f) if uplo == U_ else np.tril(f)
    prod = t @ t.T if uplo == U_ else t.T @ t
    B, ldb = _store(f, order)
    assert AB.clapack_dlauum(order, uplo, n, B, ldb) == 0
    tri = np.triu if uplo == U_ else np.tril
    assert _rel(tri(_logical(B, order)), tri(prod)) < 1e-13
    assert AB.clapack_dpotri(order, uplo, n, A, lda) == 0
    inv = tri(_logical(A, order))
    inv = inv + tri(inv, 1 if uplo == U_ else -1).T
    assert np.max(np.abs(inv @ spd - np.eye(n))) < 1e-10


@pytest.mark.parametrize("order", [CM, RM])
@pytest.mark.parametrize("trans", [NT, TR])
@pytest.mark.parametrize("m,n", [(300, 120), (120, 300)])
def test_dgels(gpu, order, trans, m, n):
    nrhs = 3
    r = _rng(6)
    a = r.uniform(-1, 1, (m, n))
    op = a if trans == NT else a.T
    rows_b, cols_x = op.shape
    b = r.uniform(-1, 1, (rows_b, nrhs))
    x_ref = np.linalg.lstsq(op, b, rcond=None)[0]  # least squares or minimum norm
    A, lda = _store(a, order)
    # B is column-major in either order, as the reference's clapack_dgels takes it
    B = np.zeros((max(m, n), nrhs), order="F")
    B[:rows_b] = b
    assert AB.clapack_dgels(order, trans, m, n, nrhs, A, lda, B, max(m, n)) == 0
    x = B[:cols_x]
    assert _rel(x, x_ref) < 1e-10


@pytest.mark.parametrize("m,n", [(60, 140), (140, 60), (100, 100)])
def test_dgelqf_is_transposed_qr(gpu, m, n):
    a = O.gegen(m, n, m, 9)[:m, :n].copy(order="F")
    tau = np.zeros(min(m, n))
    A = a.copy(order="F")
    assert AB.clapack_dgelqf(CM, m, n, A, m, tau) == 0
    qr, rtau = O.dgeqrf(np.asfortranarray(a.T))
    assert _rel(A, qr.T) < 1e-11
    assert _rel(tau, rtau) < 1e-11


@pytest.mark.parametrize("side", [L_, R_])
@pytest.mark.parametrize("trans", [NT, TR])
def test_dormqr(gpu, side, trans):
    m, k, other = 260, 200, 90
    a = O.gegen(m, k, m, 10)[:m, :k].copy(order="F")
    tau = np.zeros(k)
    qr = a.copy(order="F")
    assert AB.clapack_dgeqrf(CM, m, k, qr, m, tau) == 0
    Q = np.eye(m)   # H(0) H(1) ... H(k-1) from the reflectors, in FP64 on the host
    for i in range(k):
        v = np.zeros(m)
        v[i] = 1.0
        v[i + 1:] = qr[i + 1:, i]
        Q -= tau[i] * np.outer(Q @ v, v)
    r = _rng(11)
    c = r.uniform(-1, 1, (m, other) if side == L_ else (other, m))
    op = Q if trans == NT else Q.T
    ref = op @ c if side == L_ else c @ op
    C = c.copy(order="F")
    mm, nn = C.shape
    assert AB.ATL_dormqr(side, trans, mm, nn, k, qr, m, tau, C, mm, None, 0) == 0
    assert _rel(C, ref) < 1e-12


def _i(v):
    return ctypes.byref(ctypes.c_int(v))


def _d(v):
    return ctypes.byref(ctypes.c_double(v))


def test_f77_dgemm_and_lapack(gpu):
    lib = AB.lib()
    m, n, k = 70, 50, 40
    r = _rng(12)
    a = np.asfortranarray(r.uniform(-1, 1, (m, k)))
    b = np.asfortranarray(r.uniform(-1, 1, (k, n)))
    c = np.asfortranarray(r.uniform(-1, 1, (m, n)))
    ref = 0.5 * a @ b + 2.0 * c
    lib.dgemm_(b"N", b"N", _i(m), _i(n), _i(k), _d(0.5), AB.ptr(a), _i(m), AB.ptr(b), _i(k), _d(2.0),
               AB.ptr(c), _i(m))
    assert _rel(c, ref) < 1e-13
    # dgesv_ with 1-based pivots, against clapack_dgesv
    nn = 120
    a0 = O.gegen(nn, nn, nn, 13)[:nn, :nn]
    b0 = r.uniform(-1, 1, (nn, 2))
    a1, b1 = a0.copy(order="F"), b0.copy(order="F")
    a2, b2 = a0.copy(order="F"), b0.copy(order="F")
    p1 = np.zeros(nn, np.int32)
    p2 = np.zeros(nn, np.int32)
    info = ctypes.c_int(-99)
    lib.dgesv_(_i(nn), _i(2), AB.ptr(a1), _i(nn), AB.ptr(p1), AB.ptr(b1), _i(nn), ctypes.byref(info))
    assert info.value == 0
    assert AB.clapack_dgesv(CM, nn, 2, a2, nn, p2, b2, nn) == 0
    np.testing.assert_array_equal(p1, p2 + 1)
    np.testing.assert_array_equal(a1, a2)
    assert _rel(b1, b2) < 1e-14
    # dgetrs_ takes the 1-based pivots back
    b3 = b0.copy(order="F")
    lib.dgetrs_(b"N", _i(nn), _i(2), AB.ptr(a1), _i(nn), AB.ptr(p1), AB.ptr(b3), _i(nn), ctypes.byref(info))
    assert info.value == 0 and _rel(b3, b2) < 1e-14
    # dpotrf_ / dpotri_
    spd = O.spd_matrix(80, 3)
    f = spd.copy(order="F")
    lib.dpotrf_(b"L", _i(80), AB.ptr(f), _i(80), ctypes.byref(info))
    assert info.value == 0
    lib.dpotri_(b"l", _i(80), AB.ptr(f), _i(80), ctypes.byref(info))
    inv = np.tril(f) + np.tril(f, -1).T
    assert info.value == 0 and np.max(np.abs(inv @ spd - np.eye(80))) < 1e-10
    # dgels_ workspace query, then the solve
    work = np.zeros(1)
    a4 = np.asfortranarray(r.uniform(-1, 1, (100, 30)))
    b4 = np.asfortranarray(r.uniform(-1, 1, (100, 1)))
    x_ref = np.linalg.lstsq(a4, b4, rcond=None)[0]
    lib.dgels_(b"N", _i(100), _i(30), _i(1), AB.ptr(a4), _i(100), AB.ptr(b4), _i(100), AB.ptr(work), _i(-1),
               ctypes.byref(info))
    lw = int(work[0])
    work = np.zeros(lw)
    lib.dgels_(b"N", _i(100), _i(30), _i(1), AB.ptr(a4), _i(100), AB.ptr(b4), _i(100), AB.ptr(work), _i(lw),
               ctypes.byref(info))
    assert info.value == 0 and _rel(b4[:30], x_ref) < 1e-10


def test_f77_argument_errors_report_positions(gpu):
    lib = AB.lib()
    info = ctypes.c_int(0)
    a = np.zeros((4, 4), order="F")
    ipiv = np.zeros(4, np.int32)
    lib.dgetrf_(_i(4), _i(4), AB.ptr(a), _i(2), AB.ptr(ipiv), ctypes.byref(info))   # lda < m
    assert info.value == -4
    lib.dpotrf_(b"X", _i(4), AB.ptr(a), _i(4), ctypes.byref(info))
    assert info.value == -1
