"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every symbol include/atlas_b200.h declares, and rejects bad arguments at the
positions the reference's interface layer reports (interfaces/blas/C/src/
cblas_*.c, interfaces/lapack/C/src/clapack_*.c) -- in return mode, before any
device work is issued."""
import ctypes

import numpy as np
import pytest

import atlas_b200 as AB

CM, RM = AB.CblasColMajor, AB.CblasRowMajor
N_, T_ = AB.CblasNoTrans, AB.CblasTrans
U_, L_ = AB.CblasUpper, AB.CblasLower
NU, UN = AB.CblasNonUnit, AB.CblasUnit
LE, RI = AB.CblasLeft, AB.CblasRight


def test_library_exports_every_declared_symbol(atl):
    lib = ctypes.CDLL(AB.LIB_PATH)
    names = AB.declared_symbols()
    assert "cblas_dgemm" in names and "clapack_dgetrf" in names and "ATL_dgeqrf" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_error_mode_switch(atl):
    assert atl.atlb_get_error_mode() == 1


def _pos(call):
    call()
    return -AB.atlb_last_error()


@pytest.mark.parametrize("args,pos", [
    ((CM, N_, N_, -1, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4), 4),
    ((CM, N_, N_, 4, -1, 4, 1.0, None, 4, None, 4, 0.0, None, 4), 5),
    ((CM, N_, N_, 4, 4, -1, 1.0, None, 4, None, 4, 0.0, None, 4), 6),
    ((CM, N_, N_, 4, 4, 4, 1.0, None, 3, None, 4, 0.0, None, 4), 9),
    ((CM, N_, N_, 4, 4, 4, 1.0, None, 4, None, 3, 0.0, None, 4), 11),
    ((CM, N_, N_, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 3), 14),
    ((CM, 999, N_, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4), 2),
    ((CM, N_, 999, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4), 3),
    ((RM, N_, N_, 4, 5, 6, 1.0, None, 5, None, 5, 0.0, None, 5), 9),   # row-major: lda >= K
    ((RM, N_, N_, 4, 5, 6, 1.0, None, 6, None, 4, 0.0, None, 5), 11),  # ldb >= N
    ((7, N_, N_, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4), 1),
    ((CM, N_, N_, -1, 4, 4, 1.0, None, 0, None, 4, 0.0, None, 4), 4),  # first bad position wins
])
def test_dgemm_argument_positions(atl, args, pos):
    assert _pos(lambda: AB.cblas_dgemm(*args)) == pos


def test_trsm_syrk_argument_positions(atl):
    assert _pos(lambda: AB.cblas_dtrsm(CM, 5, U_, N_, NU, 4, 4, 1.0, None, 4, None, 4)) == 2
    assert _pos(lambda: AB.cblas_dtrsm(CM, LE, 5, N_, NU, 4, 4, 1.0, None, 4, None, 4)) == 3
    assert _pos(lambda: AB.cblas_dtrsm(CM, LE, U_, 5, NU, 4, 4, 1.0, None, 4, None, 4)) == 4
    assert _pos(lambda: AB.cblas_dtrsm(CM, LE, U_, N_, 5, 4, 4, 1.0, None, 4, None, 4)) == 5
    assert _pos(lambda: AB.cblas_dtrsm(CM, LE, U_, N_, NU, -4, 4, 1.0, None, 4, None, 4)) == 6
    assert _pos(lambda: AB.cblas_dtrsm(CM, RI, U_, N_, NU, 4, 6, 1.0, None, 4, None, 4)) == 10
    assert _pos(lambda: AB.cblas_dtrsm(CM, LE, U_, N_, NU, 4, 4, 1.0, None, 4, None, 3)) == 12
    assert _pos(lambda: AB.cblas_dsyrk(CM, 5, N_, 4, 4, 1.0, None, 4, 0.0, None, 4)) == 2
    assert _pos(lambda: AB.cblas_dsyrk(CM, U_, N_, -4, 4, 1.0, None, 4, 0.0, None, 4)) == 4
    assert _pos(lambda: AB.cblas_dsyrk(CM, U_, T_, 4, 6, 1.0, None, 5, 0.0, None, 4)) == 8
    assert _pos(lambda: AB.cblas_dsyrk(CM, U_, N_, 4, 4, 1.0, None, 4, 0.0, None, 3)) == 11


def test_lapack_argument_returns(atl):
    assert AB.clapack_dgetrf(CM, -1, 4, None, 4, None) == -2
    assert AB.clapack_dgetrf(CM, 4, 4, None, 3, None) == -6
    assert AB.clapack_dgetrf(RM, 4, 6, None, 5, None) == -6
    assert AB.clapack_dgetrs(CM, 999, 4, 1, None, 4, None, None, 4) == -2
    assert AB.clapack_dgetrs(CM, N_, 4, 1, None, 4, None, None, 3) == -9
    assert AB.clapack_dgesv(CM, 4, 1, None, 3, None, None, 4) == -5
    assert AB.clapack_dgesv(CM, 4, 1, None, 4, None, None, 3) == -8
    assert AB.clapack_dpotrf(CM, 5, 4, None, 4) == -2
    assert AB.clapack_dpotrf(CM, U_, 4, None, 3) == -5
    assert AB.clapack_dpotrs(CM, U_, 4, -1, None, 4, None, 4) == -4
    assert AB.clapack_dposv(CM, L_, 4, 1, None, 4, None, 2) == -8
    assert AB.clapack_dgeqrf(CM, 4, -1, None, 4, None) == -3
    assert AB.clapack_dgeqrf(RM, 4, 6, None, 5, None) == -5


def test_geqrf_workspace_query(atl):
    w = np.zeros(1)
    assert AB.ATL_dgeqrf(100, 40, None, 100, None, w, -1) == 0
    nb = 32
    assert w[0] == 40 * nb + nb * nb + 100


def test_quick_returns_touch_nothing(atl):
    # M == 0 / N == 0 return before any device work (src/blas/ammm/ATL_ammm.c quick return)
    c = np.full((3, 3), 7.0, order="F")
    AB.cblas_dgemm(CM, N_, N_, 0, 3, 3, 1.0, c, 3, c, 3, 0.0, c, 3)
    assert np.all(c == 7.0)
    assert AB.clapack_dgetrf(CM, 0, 5, c, 1, None) == 0
