"""Parity at the benchmark configurations' full sizes, through the C ABI:

* DGEMM C = 1.0*A*B + 0.0*C, NN, M = N = K = 2048, A and B uniform[-1,1]:
  the l3blastst residual against the oracle (bin/l3blastst.c:728-731, < 50);
* dgetrf + dgetrs at N = 8192 on A = G/sqrt(N) + 4I with 16 right-hand sides
  uniform[-1,1]: ipiv identical to the oracle's restatement of ATLAS's
  recursive getrfC (pinned to the reference's own getrf by
  tests/test_oracle.py), the factors and solutions within rounding of the
  oracle's, and the lutst residual (bin/lutst.c:244-245, <= 100);
* dpotrf + dpotrs at N = 8192 on A = G G^T / N + I: the llttst residual
  (bin/llttst.c:344, <= 100) and the solve's slvtst residual;
* dgeqrf of a 16384 x 8192 Gaussian matrix: the qrtst residual
  ||A - Q R||_1 / (||A||_1 eps min(M, N)) (bin/qrtst.c:1293-1295, <= 100),
  Q applied to R in FP64 on the GPU from the returned reflectors and tau
  (compact WY blocks, independent of the library's own larft / larfb);
* mixed dsposv at N = 8192 (SPD, cond 1e2): normwise backward error
  <= N * 2^-53.

Residuals that need O(N^3) work are computed on the GPU in FP64 with torch
(cuBLAS) -- independent of the library's kernels."""
import numpy as np
import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu
EPS = 2.0 ** -52
CM = AB.CblasColMajor


def _t(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _norm1(t):
    return t.abs().sum(dim=0).max().item()


def test_dgemm_2048_l3blastst_residual(gpu, orc):
    n = 2048
    a = orc.uniform((n, n), 101)
    b = orc.uniform((n, n), 102)
    c = np.zeros((n, n), order="F")
    AB.cblas_dgemm(CM, 111, 111, n, n, n, 1.0, a, n, b, n, 0.0, c, n)
    c0 = np.zeros((n, n), order="F")
    r = orc.resid_gemm(111, 111, n, n, n, 1.0, a, b, 0.0, c0, c)
    assert r < 50.0, r


def test_getrf_getrs_8192_matches_oracle(gpu, orc):
    import torch
    n, nrhs = 8192, 16
    a0 = orc.lu_matrix(n, 2024)
    b0 = orc.uniform((n, nrhs), 2025)
    lu = a0.copy(order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    assert AB.clapack_dgetrf(CM, n, n, lu, n, ipiv) == 0
    x = b0.copy(order="F")
    assert AB.clapack_dgetrs(CM, 111, n, nrhs, lu, n, ipiv, x, n) == 0
    # the oracle: ATLAS's recursion on the host cores
    rlu, ripiv, rinfo = orc.dgetrf(a0.copy(order="F"))
    assert rinfo == 0
    np.testing.assert_array_equal(ipiv, ripiv)
    assert np.max(np.abs(lu - rlu)) <= 1e-11 * np.max(np.abs(rlu))
    rx = orc.dgetrs(111, rlu, ripiv, b0.copy(order="F"))
    assert np.max(np.abs(x - rx)) <= 1e-11 * max(1.0, np.max(np.abs(rx)))
    # lutst residual ||P A - L U||_1 / (||A||_1 eps n), in FP64 on the GPU (here P = I)
    assert np.array_equal(ipiv, np.arange(n, dtype=np.int32))
    LU = _t(lu.T).t()                 # logical matrix
    L = torch.tril(LU, -1) + torch.eye(n, dtype=torch.float64, device="cuda")
    U = torch.triu(LU)
    A = _t(a0.T).t()
    r = _norm1(A - L @ U) / (_norm1(A) * EPS * n)
    assert r <= 100.0, r
    # slvtst-style backward check of the solve
    X = _t(x.T).t()
    B = _t(b0.T).t()
    res = (A @ X - B).abs().max().item() / (_norm1(A) * X.abs().max().item() * n * EPS)
    assert res <= 100.0, res


def test_potrf_potrs_8192_residuals(gpu, orc):
    import torch
    n, nrhs = 8192, 16
    g = torch.Generator(device="cuda")
    g.manual_seed(77)
    G = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    A = G @ G.t() / n + torch.eye(n, dtype=torch.float64, device="cuda")
    A = 0.5 * (A + A.t())
    for uplo in (AB.CblasLower, AB.CblasUpper):
        f = A.clone()                           # symmetric: row- and column-major agree
        dinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert AB.atlb_dpotrf_dev(uplo, n, f, n, dinfo) == 0
        AB.atlb_sync()
        assert int(dinfo.item()) == 0
        F = f.t()                               # logical matrix of the column-major buffer
        T = torch.tril(F) if uplo == AB.CblasLower else torch.triu(F)
        R = A - (T @ T.t() if uplo == AB.CblasLower else T.t() @ T)
        r = _norm1(R) / (_norm1(A) * EPS * n)
        assert r <= 100.0, (uplo, r)
        b = torch.rand(nrhs, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1  # col-major n x nrhs
        x = b.clone()
        assert AB.atlb_dpotrs_dev(uplo, n, nrhs, f, n, x, n) == 0
        AB.atlb_sync()
        res = (A @ x.t() - b.t()).abs().max().item() / (_norm1(A) * x.abs().max().item() * n * EPS)
        assert res <= 100.0, (uplo, res)


def _apply_q(QR, tau, X, nb=256):
    """X <- Q X with Q = H_0 H_1 ... H_{k-1} from geqrf's reflectors (unit lower
    trapezoid of QR) and tau: blocks of nb reflectors as I - V T V^T (T from
    the forward column-wise recurrence), applied last block first."""
    import torch
    m, k = QR.shape[0], tau.shape[0]
    for j0 in reversed(range(0, k, nb)):
        j1 = min(k, j0 + nb)
        w = j1 - j0
        V = torch.tril(QR[j0:, j0:j1], -1)
        V[:w, :w] += torch.eye(w, dtype=QR.dtype, device=QR.device)
        Gm = V.t() @ V
        T = torch.zeros(w, w, dtype=QR.dtype, device=QR.device)
        for i in range(w):
            T[i, i] = tau[j0 + i]
            if i:
                T[:i, i] = -tau[j0 + i] * (T[:i, :i] @ Gm[:i, i])
        X[j0:] -= V @ (T @ (V.t() @ X[j0:]))
    return X


def test_geqrf_16384x8192_qrtst_residual(gpu):
    import torch
    m, n = 16384, 8192
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    A = torch.randn(m, n, dtype=torch.float64, device="cuda", generator=g)
    buf = A.t().contiguous()                  # column-major storage of A
    tau = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert AB.atlb_dgeqrf_dev(m, n, buf, m, tau) == 0
    AB.atlb_sync()
    QR = buf.t()
    assert bool(((tau == 0) | ((tau >= 1) & (tau <= 2))).all())
    X = torch.triu(QR).contiguous()
    X = _apply_q(QR, tau, X)
    r = _norm1(A - X) / (_norm1(A) * EPS * n)
    assert r <= 100.0, r


def test_mixed_dsposv_8192_backward_error(gpu, orc):
    import torch
    n = 8192
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    Q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    s = torch.logspace(0, -2, n, dtype=torch.float64, device="cuda")
    A = (Q * s) @ Q.t()
    A = 0.5 * (A + A.t())
    b = torch.rand(1, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a_h = A.cpu().numpy().copy(order="F")
    b_h = b.cpu().numpy().T.copy(order="F")
    x_h = np.zeros((n, 1), order="F")
    it = np.zeros(1, dtype=np.int32)
    info = AB.atlb_dsposv(AB.CblasLower, n, 1, a_h, n, b_h, n, x_h, n, AB.PREC_TF32X3, it)
    assert info == 0
    assert it[0] >= 0, it[0]       # converged without the FP64 fallback
    X = _t(x_h.T).t()
    r = (A @ X - b.t()).abs().max().item()
    bwd = r / (A.abs().sum(dim=1).max().item() * X.abs().max().item() + b.abs().max().item())
    assert bwd <= n * 2.0 ** -53, bwd
