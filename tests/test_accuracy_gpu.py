"""Accuracy at sizes beyond the tester's: the triangular solves of getrs (the
one-launch path for few right-hand sides and the TRSM path) against scipy's
FP64 substitution on the same factors, and the getrf factors against
scipy's LU (same pivots on random matrices).  The tester residuals
(bin/slvtst.c, bin/lutst.c, pass <= 100) are loose enough to hide an
accuracy loss of a few orders of magnitude; these bounds are tight."""
import numpy as np
import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu

NOTRANS, TRANS = 111, 112


def _factors(n, seed):
    rng = np.random.default_rng(seed)
    L = np.tril(rng.uniform(-1, 1, (n, n)), -1) / np.sqrt(n) + np.eye(n)
    U = np.triu(rng.uniform(-1, 1, (n, n))) / np.sqrt(n) + np.diag(rng.uniform(1, 2, n))
    return L, U


@pytest.mark.parametrize("n,nrhs,trans", [(1000, 1, NOTRANS), (4096, 1, NOTRANS), (4096, 3, NOTRANS),
                                          (4096, 8, NOTRANS), (3000, 1, TRANS), (2500, 12, NOTRANS),
                                          (2048, 29, TRANS), (1500, 32, NOTRANS), (1500, 33, NOTRANS),
                                          (8192, 1, NOTRANS)])
def test_getrs_matches_substitution(gpu, n, nrhs, trans):
    import scipy.linalg as sl
    import torch
    L, U = _factors(n, n + nrhs)
    lu = np.tril(L, -1) + U                                     # packed factors, ipiv = identity
    dlu = torch.tensor(np.asfortranarray(lu).T.copy(), device="cuda")   # column-major storage
    ipiv = torch.arange(n, dtype=torch.int32, device="cuda")
    rng = np.random.default_rng(7)
    b = rng.uniform(-1, 1, (n, nrhs))
    db = torch.tensor(np.asfortranarray(b).T.copy(), device="cuda")
    assert AB.atlb_dgetrs_dev(trans, n, nrhs, dlu, n, ipiv, db, n) == 0
    AB.atlb_sync()
    x = db.cpu().numpy().T
    if trans == NOTRANS:
        ref = sl.solve_triangular(U, sl.solve_triangular(L, b, lower=True, unit_diagonal=True))
    else:
        ref = sl.solve_triangular(L.T, sl.solve_triangular(U.T, b, lower=True), unit_diagonal=True)
    err = np.abs(x - ref).max() / np.abs(ref).max()
    assert err < 1e-13, err


@pytest.mark.parametrize("n", [2048, 4096])
def test_getrf_factors_match_scipy(gpu, n):
    import scipy.linalg as sl
    import torch
    rng = np.random.default_rng(n)
    a = rng.uniform(-1, 1, (n, n))
    da = torch.tensor(np.asfortranarray(a).T.copy(), device="cuda")
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert AB.atlb_dgetrf_dev(n, n, da, n, ipiv, info) == 0
    AB.atlb_sync()
    assert int(info.item()) == 0
    lu, piv = sl.lu_factor(a)
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv)
    got = da.cpu().numpy().T
    err = np.abs(got - lu).max() / np.abs(lu).max()
    assert err < 1e-11, err
    # backward error of a solve with these factors, next to LAPACK's own
    b = rng.uniform(-1, 1, n)
    db = torch.tensor(b, device="cuda")
    assert AB.atlb_dgetrs_dev(NOTRANS, n, 1, da, n, ipiv, db, n) == 0
    AB.atlb_sync()
    x = db.cpu().numpy()

    def berr(x):
        return np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())
    ours, ref = berr(x), berr(sl.lu_solve((lu, piv), b))
    assert ours < 10 * ref + 1e-17, (ours, ref)
