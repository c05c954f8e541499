"""ctypes front end of the CPU oracle (oracle/atl_oracle.c) and of the
reference's own C BLAS and LAPACK compiled into oracle/_ref/ by
oracle/build_ref.sh.

Test infrastructure only: imported by tests/, the smoke check and the CPU
baseline leg of bench.py -- never by the library.  Arrays are numpy,
column-major (order='F'), float64 unless noted.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libatlref.so")
REF_LAPACK_LIB = os.path.join(HERE, "_ref", "libatlref_lapack.so")

NoTrans, Trans = 111, 112
Upper, Lower = 121, 122
NonUnit, Unit = 131, 132
Left, Right = 141, 142

_I, _D, _F, _P, _L, _U64 = (ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p,
                            ctypes.c_int64, ctypes.c_uint64)

_SIGS = {
    "orc_set_threads": (None, [_I]),
    "orc_srand": (None, [_I]),
    "orc_rand": (_I, []),
    "orc_gegen": (None, [_I, _I, _P, _I, _I]),
    "orc_gechkgap": (_I, [_I, _I, _P, _I]),
    "orc_fill_uniform": (None, [_L, _P, _U64, _D, _D]),
    "orc_fill_normal": (None, [_L, _P, _U64]),
    "orc_dgemm": (None, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "orc_sgemm": (None, [_I, _I, _I, _I, _I, _F, _P, _I, _P, _I, _F, _P, _I]),
    "orc_dtrsm": (None, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "orc_dtrmm": (None, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "orc_dsyrk": (None, [_I, _I, _I, _I, _D, _P, _I, _D, _P, _I]),
    "orc_dlaswp": (None, [_I, _P, _I, _I, _I, _P, _I]),
    "orc_dgetrf": (_I, [_I, _I, _P, _I, _P]),
    "orc_dgetrs": (None, [_I, _I, _I, _P, _I, _P, _P, _I]),
    "orc_dpotrf": (_I, [_I, _I, _P, _I]),
    "orc_dpotrs": (None, [_I, _I, _I, _P, _I, _P, _I]),
    "orc_dlarfg": (None, [_I, _P, _P, _P]),
    "orc_dgeqr2": (None, [_I, _I, _P, _I, _P]),
    "orc_dlarft": (None, [_I, _I, _P, _I, _P, _P, _I]),
    "orc_dlarfb_lt": (None, [_I, _I, _I, _P, _I, _P, _I, _P, _I]),
    "orc_dgeqrf": (_I, [_I, _I, _P, _I, _P, _I]),
    "orc_genrm1": (_D, [_I, _I, _P, _I]),
    "orc_resid_gemm": (_D, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I, _P, _I]),
    "orc_resid_lu": (_D, [_I, _I, _P, _I, _P, _I, _P]),
    "orc_resid_llt": (_D, [_I, _I, _P, _I, _P, _I]),
    "orc_resid_qr": (_D, [_I, _I, _P, _I, _P, _I, _P]),
    "orc_resid_slv": (_D, [_I, _I, _P, _I, _P, _I, _P, _I]),
    "orc_ddgemm": (None, [_I, _I, _I, _P, _I, _P, _I, _P, _P, _I]),
    "orc_normwise_err_dd": (_D, [_I, _I, _P, _I, _P, _P, _I]),
}

_REF_SIGS = {
    "ATL_drefgemm": (None, [_I, _I, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "ATL_srefgemm": (None, [_I, _I, _I, _I, _I, _F, _P, _I, _P, _I, _F, _P, _I]),
    "ATL_dreftrsm": (None, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "ATL_dreftrmm": (None, [_I, _I, _I, _I, _I, _I, _D, _P, _I, _P, _I]),
    "ATL_drefsyrk": (None, [_I, _I, _I, _I, _D, _P, _I, _D, _P, _I]),
}

# the reference's LAPACK entry points (src/lapack/ATL_getrf.c:8, ATL_getrs.c:8,
# ATL_potrf.c:7, ATL_potrs.c:13, ATL_geqrf.c:29), type-prefixed as a DREAL build names them
_REF_LAPACK_SIGS = {
    "ATL_dgetrf": (_I, [_I, _I, _I, _P, _I, _P]),
    "ATL_dgetrs": (None, [_I, _I, _I, _I, _P, _I, _P, _P, _I]),
    "ATL_dpotrf": (_I, [_I, _I, _I, _P, _I]),
    "ATL_dpotrs": (None, [_I, _I, _I, _I, _P, _I, _P, _I]),
    "ATL_dgeqrf": (_I, [_I, _I, _P, _I, _P, _P, _I]),
}

_orc = None
_ref = None
_ref_lapack = None


def _load(path, sigs):
    l = ctypes.CDLL(path)
    for n, (r, a) in sigs.items():
        f = getattr(l, n)
        f.restype, f.argtypes = r, a
    return l


def orc():
    """The C restatement (builds it with make on first use if missing)."""
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_LIB):
            subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
        _orc = _load(ORC_LIB, _SIGS)
    return _orc


def ref_available():
    return os.path.exists(REF_LIB)


def ref():
    """The reference's own C reference BLAS (oracle/_ref/libatlref.so)."""
    global _ref
    if _ref is None:
        _ref = _load(REF_LIB, _REF_SIGS)
    return _ref


def ref_lapack_available():
    return os.path.exists(REF_LAPACK_LIB)


def ref_lapack():
    """The reference's own LAPACK path (oracle/_ref/libatlref_lapack.so)."""
    global _ref_lapack
    if _ref_lapack is None:
        _ref_lapack = _load(REF_LAPACK_LIB, _REF_LAPACK_SIGS)
    return _ref_lapack


def ref_dgetrf(a, order=102):
    """ATL_getrf of the reference on a copy of a: (LU, ipiv, info)."""
    a = np.array(a, order="F", copy=True)
    m, n = a.shape
    if order == 101:  # row-major: the buffer holds the m x n matrix row by row
        ld = n
        buf = np.ascontiguousarray(a)
    else:
        ld = m
        buf = a
    ipiv = np.zeros(max(min(m, n), 1), dtype=np.int32)
    info = ref_lapack().ATL_dgetrf(order, m, n, buf.ctypes.data, max(ld, 1), ipiv.ctypes.data)
    out = np.asfortranarray(buf) if order == 101 else buf
    return out, ipiv[:min(m, n)], info


def ref_dgetrs(trans, lu, ipiv, b):
    b = np.array(b, order="F", copy=True)
    n = lu.shape[1]
    ref_lapack().ATL_dgetrs(102, trans, n, b.shape[1], P(lu), lu.shape[0],
                            np.ascontiguousarray(ipiv, np.int32).ctypes.data, P(b), b.shape[0])
    return b


def ref_dpotrf(uplo, a):
    a = np.array(a, order="F", copy=True)
    info = ref_lapack().ATL_dpotrf(102, uplo, a.shape[1], P(a), a.shape[0])
    return a, info


def ref_dpotrs(uplo, f, b):
    b = np.array(b, order="F", copy=True)
    ref_lapack().ATL_dpotrs(102, uplo, f.shape[1], b.shape[1], P(f), f.shape[0], P(b), b.shape[0])
    return b


def ref_dgeqrf(a):
    """ATL_geqrf of the reference (workspace query, then the factorization)."""
    a = np.array(a, order="F", copy=True)
    m, n = a.shape
    tau = np.zeros(max(min(m, n), 1))
    w = np.zeros(1)
    lib = ref_lapack()
    lib.ATL_dgeqrf(m, n, P(a), max(m, 1), P(tau), P(w), -1)
    lw = max(int(w[0]), 1)
    w = np.zeros(lw)
    info = lib.ATL_dgeqrf(m, n, P(a), max(m, 1), P(tau), P(w), lw)
    return a, tau[:min(m, n)], info


def P(a):
    """Address of a column-major array (a C-ordered 2-D array would be read transposed)."""
    if a is None:
        return None
    if a.ndim == 2 and a.shape[1] > 1 and not a.flags.f_contiguous:
        raise ValueError("oracle arrays are column-major: pass np.asfortranarray(...)")
    return a.ctypes.data


# ---------------------------------------------------------------- generators
def gegen(m, n, lda, seed):
    """ATL_gegen: M x N in an lda x N buffer, the lda gap poisoned."""
    a = np.empty((lda, max(n, 1)), order="F")
    orc().orc_gegen(m, n, P(a), lda, seed)
    return a


def gechkgap(a, m, n):
    return orc().orc_gechkgap(m, n, P(a), a.shape[0])


def uniform(shape, seed, lo=-1.0, hi=1.0):
    a = np.empty(shape, order="F")
    orc().orc_fill_uniform(a.size, P(a), seed, lo, hi)
    return a


def normal(shape, seed):
    a = np.empty(shape, order="F")
    orc().orc_fill_normal(a.size, P(a), seed)
    return a


def lu_matrix(n, seed):
    """A = G/sqrt(n) + 4 I (the factorization benchmarks' LU input)."""
    return np.asfortranarray(normal((n, n), seed) / np.sqrt(n) + 4.0 * np.eye(n))


def spd_matrix(n, seed):
    """A = G G^T / n + I."""
    g = normal((n, n), seed)
    a = np.empty((n, n), order="F")
    orc().orc_dgemm(NoTrans, Trans, n, n, n, 1.0 / n, P(g), n, P(g), n, 0.0, P(a), n)
    a += np.eye(n)
    return np.asfortranarray(0.5 * (a + a.T))


# ---------------------------------------------------------------- BLAS
def dgemm(ta, tb, m, n, k, alpha, a, b, beta, c):
    orc().orc_dgemm(ta, tb, m, n, k, alpha, P(a), a.shape[0], P(b), b.shape[0], beta, P(c), c.shape[0])
    return c


def sgemm(ta, tb, m, n, k, alpha, a, b, beta, c):
    orc().orc_sgemm(ta, tb, m, n, k, alpha, P(a), a.shape[0], P(b), b.shape[0], beta, P(c), c.shape[0])
    return c


def dtrsm(side, uplo, ta, diag, m, n, alpha, a, b):
    orc().orc_dtrsm(side, uplo, ta, diag, m, n, alpha, P(a), a.shape[0], P(b), b.shape[0])
    return b


def dtrmm(side, uplo, ta, diag, m, n, alpha, a, b):
    orc().orc_dtrmm(side, uplo, ta, diag, m, n, alpha, P(a), a.shape[0], P(b), b.shape[0])
    return b


def dsyrk(uplo, trans, n, k, alpha, a, beta, c):
    orc().orc_dsyrk(uplo, trans, n, k, alpha, P(a), a.shape[0], beta, P(c), c.shape[0])
    return c


# ---------------------------------------------------------------- LAPACK
def dgetrf(a, m=None, n=None):
    m = a.shape[0] if m is None else m
    n = a.shape[1] if n is None else n
    ipiv = np.zeros(max(min(m, n), 1), dtype=np.int32)
    info = orc().orc_dgetrf(m, n, P(a), a.shape[0], P(ipiv))
    return a, ipiv[:min(m, n)], info


def dgetrs(trans, a, ipiv, b):
    n = a.shape[1]
    orc().orc_dgetrs(trans, n, b.shape[1], P(a), a.shape[0], P(np.ascontiguousarray(ipiv, np.int32)), P(b), b.shape[0])
    return b


def dpotrf(uplo, a):
    return orc().orc_dpotrf(uplo, a.shape[1], P(a), a.shape[0])


def dpotrs(uplo, a, b):
    orc().orc_dpotrs(uplo, a.shape[1], b.shape[1], P(a), a.shape[0], P(b), b.shape[0])
    return b


def dgeqrf(a, nb=32):
    m, n = a.shape
    tau = np.zeros(max(min(m, n), 1))
    orc().orc_dgeqrf(m, n, P(a), a.shape[0], P(tau), nb)
    return a, tau[:min(m, n)]


def genrm1(a):
    return orc().orc_genrm1(a.shape[0], a.shape[1], P(a), a.shape[0])


# ---------------------------------------------------------------- residuals
def resid_gemm(ta, tb, m, n, k, alpha, a, b, beta, c0, ctst):
    """bin/l3blastst.c:728-731 (pass < 50)."""
    return orc().orc_resid_gemm(ta, tb, m, n, k, alpha, P(a), a.shape[0], P(b), b.shape[0], beta,
                                P(c0), c0.shape[0], P(ctst), ctst.shape[0])


def resid_lu(a0, lu, ipiv):
    """bin/lutst.c:244-245 (pass <= 100)."""
    m, n = a0.shape
    return orc().orc_resid_lu(m, n, P(a0), a0.shape[0], P(lu), lu.shape[0],
                              P(np.ascontiguousarray(ipiv, np.int32)))


def resid_llt(uplo, a0, f):
    """bin/llttst.c:344 (pass <= 100)."""
    return orc().orc_resid_llt(uplo, a0.shape[0], P(a0), a0.shape[0], P(f), f.shape[0])


def resid_qr(a0, qr, tau):
    """bin/qrtst.c:1293-1295 (pass <= 100)."""
    m, n = a0.shape
    return orc().orc_resid_qr(m, n, P(a0), a0.shape[0], P(qr), qr.shape[0], P(np.ascontiguousarray(tau)))


def resid_slv(a, x, xtrue):
    """bin/slvtst.c:419-441 (pass <= 100)."""
    return orc().orc_resid_slv(a.shape[0], x.shape[1], P(a), a.shape[0], P(x), x.shape[0],
                               P(xtrue), xtrue.shape[0])


def ddgemm(a, b):
    """op(A)*op(B) in double-double: returns (hi, lo)."""
    m, k = a.shape
    n = b.shape[1]
    hi = np.empty((m, n), order="F")
    lo = np.empty((m, n), order="F")
    orc().orc_ddgemm(m, n, k, P(a), a.shape[0], P(b), b.shape[0], P(hi), P(lo), m)
    return hi, lo


def normwise_err_dd(c, hi, lo):
    m, n = hi.shape
    return orc().orc_normwise_err_dd(m, n, P(c), c.shape[0], P(hi), P(lo), m)


def trddom(uplo, a, n):
    """bin/l3blastst.c:539-600: scale the strict triangle by 1/n and push the
    diagonal one unit away from zero (a diagonally dominant triangle)."""
    al = 1.0 / n
    for j in range(n):
        if uplo == Upper:
            a[:j, j] *= al
        else:
            a[j + 1:n, j] *= al
        a[j, j] += 1.0 if a[j, j] >= 0 else -1.0
    return a


def tester_seeds(ma, na, mb, nb, m, n):
    """bin/l3blastst.c:665-667."""
    return ma * na + 513 * 7 + 90, mb * nb + 127 * 50 + 77, m * n + 101 * 2 + 53
