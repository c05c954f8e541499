"""Mixed-precision solvers (FP32 / TF32 / BF16 factorization + FP64
iterative refinement): the solution reaches a normwise backward error
<= N * 2^-53 (the criterion the refinement stops on, recomputed here on the
host in FP64), A and B are left unchanged when refinement succeeds, and the
FP64 fallback engages (iter < 0) when it cannot."""
import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def kappa_matrix(n, kappa, seed):
    rng = np.random.default_rng(seed)
    q1, _ = np.linalg.qr(rng.standard_normal((n, n)))
    q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.logspace(0, -np.log10(kappa), n)
    return np.asfortranarray((q1 * s) @ q2.T)


def bwd_err(a, x, b):
    r = b - a @ x
    return np.max(np.abs(r), axis=0) / (np.max(np.sum(np.abs(a), axis=1)) * np.max(np.abs(x), axis=0)
                                        + np.max(np.abs(b), axis=0))


@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("n,nrhs", [(300, 1), (1000, 3), (700, 12)])
def test_dsgesv_kappa_1e2(gpu, prec, n, nrhs):
    a0 = kappa_matrix(n, 1e2, n + prec)
    b0 = np.asfortranarray(np.random.default_rng(5).uniform(-1, 1, (n, nrhs)))
    a, b = a0.copy(order="F"), b0.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    info = AB.atlb_dsgesv(n, nrhs, a, n, ipiv, b, n, x, n, prec, it)
    assert info == 0
    assert it[0] >= 0, f"refinement did not converge (iter={it[0]})"
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    assert np.array_equal(a, a0) and np.array_equal(b, b0)


def test_dsgesv_bf16_kappa_1e6_falls_back_or_converges(gpu):
    n = 400
    a0 = kappa_matrix(n, 1e6, 9)
    b0 = np.asfortranarray(np.random.default_rng(6).uniform(-1, 1, (n, 1)))
    a, b = a0.copy(order="F"), b0.copy(order="F")
    x = np.zeros((n, 1), order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsgesv(n, 1, a, n, ipiv, b, n, x, n, 2, it) == 0
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    if it[0] < 0:   # FP64 fallback: A holds the FP64 factors, like dgesv
        ref, rpiv, _ = O.dgetrf(a0.copy(order="F"))
        np.testing.assert_array_equal(ipiv, rpiv)


def test_dsgesv_singular(gpu):
    n = 64
    a0 = O.lu_matrix(n, 3)
    a0[:, 10] = 0.0
    x = np.zeros((n, 1), order="F")
    b = np.ones((n, 1), order="F")
    it = np.zeros(1, dtype=np.int32)
    ipiv = np.zeros(n, dtype=np.int32)
    assert AB.atlb_dsgesv(n, 1, a0.copy(order="F"), n, ipiv, b, n, x, n, 1, it) == 11
    assert it[0] == -3


@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("uplo", [121, 122])
def test_dsposv(gpu, prec, uplo):
    n, nrhs = 500, 2
    g = np.random.default_rng(prec + uplo).standard_normal((n, n))
    a0 = np.asfortranarray(g @ g.T / n + np.eye(n))
    b0 = np.asfortranarray(np.random.default_rng(1).uniform(-1, 1, (n, nrhs)))
    a = a0.copy(order="F")
    tri = np.triu(np.ones((n, n), bool), 1) if uplo == 122 else np.tril(np.ones((n, n), bool), -1)
    a[tri] = np.nan       # the unreferenced triangle must not be read
    a_in = a.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsposv(uplo, n, nrhs, a, n, b0, n, x, n, prec, it) == 0
    assert it[0] >= 0
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    np.testing.assert_array_equal(np.isnan(a), np.isnan(a_in))


@pytest.mark.parametrize("prec", [0, 1, 3])
@pytest.mark.parametrize("n,nrhs", [(512, 1), (1001, 2), (258, 9)])
def test_dsgesv_rbt_result_is_right_either_way(gpu, prec, n, nrhs):
    """LU without pivoting after a depth-2 butterfly can grow elements by
    orders of magnitude on dense random matrices (here Q1 diag(s) Q2^T), so
    refinement may not converge; the solver must then fall back (iter = -31,
    LAPACK dsgesv's 'no convergence') and still return the FP64 solution."""
    a0 = kappa_matrix(n, 1e2, 3 * n + prec)
    b0 = np.asfortranarray(np.random.default_rng(7).uniform(-1, 1, (n, nrhs)))
    a, b = a0.copy(order="F"), b0.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsgesv_ex(n, nrhs, a, n, ipiv, b, n, x, n, prec, 1, it) == 0
    assert it[0] >= 0 or it[0] == -31, it[0]
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    if it[0] >= 0:
        assert np.array_equal(a, a0) and np.array_equal(b, b0)


@pytest.mark.parametrize("prec", [0, 3])
@pytest.mark.parametrize("n,nrhs", [(512, 1), (1001, 2), (258, 9)])
def test_dsgesv_rbt_converges_without_pivoting_needs(gpu, prec, n, nrhs):
    """On the factorization benchmark's matrix class (G/sqrt(n) + 4I, pivots
    not needed) the butterfly + no-pivot FP32-accurate factorization refines
    to the FP64 criterion."""
    rng = np.random.default_rng(n + prec)
    a0 = np.asfortranarray(rng.standard_normal((n, n)) / np.sqrt(n) + 4 * np.eye(n))
    b0 = np.asfortranarray(rng.uniform(-1, 1, (n, nrhs)))
    a, b = a0.copy(order="F"), b0.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsgesv_ex(n, nrhs, a, n, ipiv, b, n, x, n, prec, 1, it) == 0
    assert it[0] >= 0, it[0]
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    assert np.array_equal(a, a0) and np.array_equal(b, b0)


def test_dsgesv_rbt_matrix_without_pivot_needs(gpu):
    # a matrix that defeats LU without pivoting (zero leading entry) is handled
    n = 64
    a0 = O.lu_matrix(n, 11)
    a0[0, 0] = 0.0
    b0 = np.ones((n, 1), order="F")
    x = np.zeros((n, 1), order="F")
    it = np.zeros(1, dtype=np.int32)
    ipiv = np.zeros(n, dtype=np.int32)
    assert AB.atlb_dsgesv_ex(n, 1, a0.copy(order="F"), n, ipiv, b0, n, x, n, 3, 1, it) == 0
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)


@pytest.mark.parametrize("n", [1024, 3000])
def test_dsgesv_bf16_converges_by_gmres_ir(gpu, n):
    """BF16 factors leave u_bf16 * kappa * growth near 1 even at kappa = 1e2,
    where plain refinement stalls: the GMRES-IR corrections (FP64 GMRES
    preconditioned by the BF16 factors) still reach N * 2^-53 without the FP64
    fallback, and A and B stay unchanged."""
    a0 = kappa_matrix(n, 1e2, 31 + n)
    b0 = np.asfortranarray(np.random.default_rng(7).uniform(-1, 1, (n, 1)))
    a, b = a0.copy(order="F"), b0.copy(order="F")
    x = np.zeros((n, 1), order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsgesv(n, 1, a, n, ipiv, b, n, x, n, 2, it) == 0
    assert it[0] >= 0, f"no convergence (iter={it[0]})"
    assert AB.atlb_mixed_krylov_steps() > 0
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    assert np.array_equal(a, a0) and np.array_equal(b, b0)


@pytest.mark.parametrize("prec", [0, 3])
def test_dsgesv_kappa_1e6_gmres_ir_corrections(gpu, prec):
    """mixed_krylov = 2: every refinement step is a GMRES-IR correction (FP64
    GMRES preconditioned by the FP32 factors); at kappa = 1e6 it converges on
    3 right-hand sides at once, in fewer outer steps than plain refinement
    (mixed_krylov = 0) takes, to the same criterion."""
    n, nrhs = 1500, 3
    a0 = kappa_matrix(n, 1e6, 77 + prec)
    b0 = np.asfortranarray(np.random.default_rng(8).uniform(-1, 1, (n, nrhs)))
    steps = {}
    try:
        for mode in (2, 0):
            assert AB.atlb_tune_set("mixed_krylov", mode) == mode
            x = np.zeros((n, nrhs), order="F")
            ipiv = np.zeros(n, dtype=np.int32)
            it = np.zeros(1, dtype=np.int32)
            assert AB.atlb_dsgesv(n, nrhs, a0.copy(order="F"), n, ipiv, b0.copy(order="F"), n, x, n, prec, it) == 0
            assert it[0] >= 0, f"mode {mode}: no convergence (iter={it[0]})"
            assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
            steps[mode] = (int(it[0]), AB.atlb_mixed_krylov_steps())
    finally:
        AB.atlb_tune_set("mixed_krylov", 1)
    assert steps[2][1] > 0 and steps[0][1] == 0
    assert steps[2][0] <= steps[0][0]


def test_dsposv_bf16_gmres_ir(gpu):
    n = 1200
    rng = np.random.default_rng(12)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    a0 = np.asfortranarray((q * np.logspace(0, -2, n)) @ q.T)
    a0 = np.asfortranarray(0.5 * (a0 + a0.T))
    b0 = np.asfortranarray(rng.uniform(-1, 1, (n, 2)))
    x = np.zeros((n, 2), order="F")
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsposv(AB.CblasLower, n, 2, a0.copy(order="F"), n, b0.copy(order="F"), n, x, n, 2, it) == 0
    assert it[0] >= 0, f"no convergence (iter={it[0]})"
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)


@pytest.mark.parametrize("n,nrhs,pinned,lda,prec", [(2148, 1, False, 2151, 3), (4096, 2, True, 4096, 3),
                                                    (2304, 12, False, 2304, 0)])
def test_dsgesv_host_input_factored_while_copied(gpu, n, nrhs, pinned, lda, prec):
    """A host A of order >= 2048 is factored while it is copied (column
    segments N/16, N/8, N/4, N/2, N: each later segment is converted through the
    interchanges to its left and updated in two large operations): the
    solution meets the same bound as with A on the device, in about the same
    number of steps, and A is left unchanged.  2148 leaves a ragged last
    block column (with a leading dimension above the order); the pinned case
    is the asynchronous copy; FP32 factors with 12 right-hand sides take the
    SIMT products and the blocked solves."""
    import torch
    a0 = kappa_matrix(n, 1e2, n)
    b0 = np.asfortranarray(np.random.default_rng(9).uniform(-1, 1, (n, nrhs)))
    ipiv = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    # host input (column-major storage, leading dimension lda)
    if pinned:
        a = torch.empty((n, n), dtype=torch.float64).pin_memory()
        a.copy_(torch.from_numpy(np.ascontiguousarray(a0.T)))
    else:
        a = np.zeros((lda, n), order="F")
        a[:n, :] = a0
    b = b0.copy(order="F")
    x = np.zeros((n, nrhs), order="F")
    assert AB.atlb_dsgesv_ex(n, nrhs, a, lda, ipiv, b, n, x, n, prec, 0, it) == 0
    it_host = int(it[0])
    assert it_host >= 0
    assert np.all(bwd_err(a0, x, b0) <= n * 2.0 ** -53)
    a_after = a.numpy().T if pinned else a[:n, :]
    assert np.array_equal(a_after, a0)
    # the same system with A on the device (factored after one whole copy)
    da = torch.from_numpy(np.ascontiguousarray(a0.T)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b0.T)).cuda()
    dx = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    dpiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert AB.atlb_dsgesv_ex(n, nrhs, da, n, dpiv, db, n, dx, n, prec, 0, it) == 0
    assert it[0] >= 0 and abs(it_host - int(it[0])) <= 1
    xd = dx.cpu().numpy().T
    assert np.all(bwd_err(a0, xd, b0) <= n * 2.0 ** -53)


@pytest.mark.parametrize("zero_col", [100, 400, 700, 2100])
def test_dsgesv_host_input_singular_in_each_segment(gpu, zero_col):
    """A zero column in any segment of the streamed factorization (2148:
    [0, 256), [256, 512), [512, 1024), [1024, 2148)) reports its position
    through the segments' info and pivot offsets: the FP32 factorization
    fails, the FP64 one finds the same column, info = column + 1."""
    n = 2148
    a0 = np.asfortranarray(np.random.default_rng(3).uniform(-1, 1, (n, n)))
    a0[:, zero_col] = 0.0
    x = np.zeros((n, 1), order="F")
    b = np.ones((n, 1), order="F")
    it = np.zeros(1, dtype=np.int32)
    ipiv = np.zeros(n, dtype=np.int32)
    assert AB.atlb_dsgesv_ex(n, 1, a0.copy(order="F"), n, ipiv, b, n, x, n, 3, 0, it) == zero_col + 1
    assert it[0] == -3
