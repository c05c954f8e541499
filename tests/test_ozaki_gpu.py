"""Split-integer (Ozaki) DGEMM on the INT8 tensor cores against the
double-double oracle: with 8 slices its normwise error matches FP64 DGEMM's
(within 4x), fewer slices are monotonically less accurate, and transposes,
alpha/beta and ragged sizes follow BLAS semantics."""
import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CM = AB.CblasColMajor


def spread(shape, seed):
    # x = u * 2^e, u ~ U[-1,1], e ~ U{-10..10} (the benchmark's distribution)
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.uniform(-1, 1, shape) * np.exp2(rng.integers(-10, 11, shape)))


@pytest.mark.parametrize("m,n,k", [(256, 256, 1024), (300, 130, 517), (65, 257, 2000)])
def test_ozaki_matches_fp64_error(gpu, orc, m, n, k):
    a, b = spread((m, k), 1 + m), spread((k, n), 2 + n)
    hi, lo = orc.ddgemm(a, b)
    c64 = np.zeros((m, n), order="F")
    AB.cblas_dgemm(CM, 111, 111, m, n, k, 1.0, a, m, b, k, 0.0, c64, m)
    e64 = orc.normwise_err_dd(c64, hi, lo)
    errs = {}
    for s in (5, 6, 7, 8):
        c = np.zeros((m, n), order="F")
        assert AB.atlb_dgemm_ozaki(111, 111, m, n, k, 1.0, a, m, b, k, 0.0, c, m, s) == 0
        errs[s] = orc.normwise_err_dd(c, hi, lo)
    assert errs[8] <= 4 * e64 + 1e-17, (errs, e64)
    assert errs[5] > errs[6] > errs[7] >= errs[8] * 0.5, errs


@pytest.mark.parametrize("ta,tb", [(111, 112), (112, 111), (112, 112)])
def test_ozaki_transposes_alpha_beta(gpu, orc, ta, tb):
    m, n, k = 150, 90, 333
    a = spread((m, k) if ta == 111 else (k, m), 3)
    b = spread((k, n) if tb == 111 else (n, k), 4)
    c0 = spread((m, n), 5)
    c = c0.copy(order="F")
    assert AB.atlb_dgemm_ozaki(ta, tb, m, n, k, -0.5, a, a.shape[0], b, b.shape[0], 2.0, c, m, 8) == 0
    ref = -0.5 * ((a if ta == 111 else a.T) @ (b if tb == 111 else b.T)) + 2.0 * c0
    err = np.linalg.norm(c - ref) / np.linalg.norm(ref)
    assert err < 1e-14


def test_ozaki_zero_rows_and_exact_small_integers(gpu):
    m, n, k = 40, 33, 70
    a = np.asfortranarray(np.random.default_rng(0).integers(-50, 50, (m, k)).astype(np.float64))
    a[5, :] = 0.0
    b = np.asfortranarray(np.random.default_rng(1).integers(-50, 50, (k, n)).astype(np.float64))
    c = np.zeros((m, n), order="F")
    assert AB.atlb_dgemm_ozaki(111, 111, m, n, k, 1.0, a, m, b, k, 0.0, c, m, 3) == 0
    np.testing.assert_array_equal(c, a @ b)   # small integers are exact
