"""Parity of the GPU level-3 BLAS with the reference: the reference's own C
BLAS outputs (tests/golden/ref_blas.npz) and the oracle, through the C ABI
with host buffers (the drop-in path), checked by bin/l3blastst.c's residual
(< 50) plus an elementwise tolerance, with the lda gaps checked for stray
writes (ATL_gechkgap)."""
import os

import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_blas.npz")
CM, RM = AB.CblasColMajor, AB.CblasRowMajor
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_dgemm_golden_cases(gpu, orc, gold):
    for i in range(int(gold["counts"][0])):
        m, n, k, ta, tb, alpha, beta = gold[f"gemm{i}"]
        m, n, k, ta, tb = int(m), int(n), int(k), int(ta), int(tb)
        a, b = gold[f"gemm{i}_A"], gold[f"gemm{i}_B"]
        c0 = gold[f"gemm{i}_C0"]
        c = np.array(c0, order="F")
        AB.cblas_dgemm(CM, ta, tb, m, n, k, alpha, a, a.shape[0], b, b.shape[0], beta, c, c.shape[0])
        ref = gold[f"gemm{i}_C"]
        r = orc.resid_gemm(ta, tb, m, n, k, alpha, a, b, beta, c0, c)
        assert r < 50.0, f"case {i}: l3blastst residual {r}"
        assert np.max(np.abs(c[:m, :n] - ref[:m, :n])) <= 1e-13 * max(1, k), f"case {i}"
        assert orc.gechkgap(c, m, n) == 0


@pytest.mark.parametrize("ta", [111, 112])
@pytest.mark.parametrize("tb", [111, 112])
@pytest.mark.parametrize("m,n,k", [(129, 257, 95), (300, 200, 513), (1, 130, 17), (128, 128, 16)])
def test_dgemm_vs_oracle(gpu, orc, ta, tb, m, n, k):
    ma, na = (m, k) if ta == 111 else (k, m)
    mb, nb = (k, n) if tb == 111 else (n, k)
    a = orc.gegen(ma, na, ma + 1, 3 + m)     # odd lda: 8-byte staging path on the host side
    b = orc.gegen(mb, nb, mb + 2, 5 + n)
    c0 = orc.gegen(m, n, m + 3, 7 + k)
    c = np.array(c0, order="F")
    AB.cblas_dgemm(CM, ta, tb, m, n, k, 0.75, a, a.shape[0], b, b.shape[0], -1.25, c, c.shape[0])
    r = orc.resid_gemm(ta, tb, m, n, k, 0.75, a, b, -1.25, c0, c)
    assert r < 50.0
    assert orc.gechkgap(c, m, n) == 0


def test_dgemm_device_pointers_unaligned_lda(gpu, orc):
    import torch
    m, n, k = 77, 65, 91
    A = torch.randn(81, k, dtype=torch.float64, device="cuda")  # lda = 81 (odd)
    B = torch.randn(k, n, dtype=torch.float64, device="cuda")
    C = torch.zeros(m, n, dtype=torch.float64, device="cuda")
    # column-major views: pass the transposed storage of row-major torch tensors
    At, Bt, Ct = A.t().contiguous(), B.t().contiguous(), C.t().contiguous()
    assert AB.atlb_dgemm_dev(111, 111, m, n, k, 1.0, At, 81, Bt, k, 0.0, Ct, m) == 0
    AB.atlb_sync()
    ref = A[:m].double() @ B
    assert torch.allclose(Ct.t(), ref, rtol=1e-12, atol=1e-12)


def test_dgemm_row_major_and_syrk_shortcut(gpu, orc):
    m, n, k = 70, 50, 40
    a = orc.uniform((m, k), 1)  # row-major M x K == col-major K x M storage
    b = orc.uniform((k, n), 2)
    A = np.ascontiguousarray(a)
    B = np.ascontiguousarray(b)
    C = np.zeros((m, n))
    AB.cblas_dgemm(RM, 111, 111, m, n, k, 1.0, A, k, B, n, 0.0, C, n)
    np.testing.assert_allclose(C, a @ b, rtol=1e-12, atol=1e-12)
    # A == B, TA != TB, beta == 0: the reference calls SYRK + reflect (cblas_dgemm.c:123-129)
    S = np.zeros((m, m), order="F")
    af = np.asfortranarray(a)
    AB.cblas_dgemm(CM, 111, 112, m, m, k, 1.0, af, m, af, m, 0.0, S, m)
    np.testing.assert_allclose(S, a @ a.T, rtol=1e-12, atol=1e-12)
    assert np.array_equal(S, S.T)


def test_dgemm_beta_zero_ignores_nan(gpu):
    c = np.full((9, 9), np.nan, order="F")
    a = np.ones((9, 9), order="F")
    AB.cblas_dgemm(CM, 111, 111, 9, 9, 9, 1.0, a, 9, a, 9, 0.0, c, 9)
    assert np.all(c == 9.0)


@pytest.mark.parametrize("ta", [111, 112])
@pytest.mark.parametrize("tb", [111, 112])
def test_sgemm_vs_oracle(gpu, orc, ta, tb):
    m, n, k = 190, 133, 257
    ma, na = (m, k) if ta == 111 else (k, m)
    mb, nb = (k, n) if tb == 111 else (n, k)
    a = np.asfortranarray(orc.uniform((ma, na), 4), dtype=np.float32)
    b = np.asfortranarray(orc.uniform((mb, nb), 5), dtype=np.float32)
    c0 = np.asfortranarray(orc.uniform((m, n), 6), dtype=np.float32)
    c = c0.copy(order="F")
    AB.cblas_sgemm(CM, ta, tb, m, n, k, 1.5, a, ma, b, mb, 0.5, c, m)
    cr = c0.copy(order="F")
    orc.sgemm(ta, tb, m, n, k, 1.5, a, b, 0.5, cr)
    # FP32 with K=257: |error| <= ~K * eps32 * sum|a||b|
    tol = 4 * k * np.finfo(np.float32).eps * (np.abs(a).max() * np.abs(b).max() * k + 1)
    assert np.max(np.abs(c - cr)) <= tol


@pytest.mark.parametrize("ta,tb", [(111, 111), (112, 112), (111, 112)])
@pytest.mark.parametrize("m,n,k", [(200, 150, 5000), (128, 128, 4096)])
def test_sgemm_split_k_vs_fp64(gpu, ta, tb, m, n, k):
    """A few output tiles with a long K: the SIMT FP32 GEMM splits K over the
    grid (partial products summed by a second pass) -- alpha, beta and the
    transposes still apply, to FP32 accuracy against an FP64 product."""
    rng = np.random.default_rng(m + n + k + ta + tb)
    ma, na = (m, k) if ta == 111 else (k, m)
    mb, nb = (k, n) if tb == 111 else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ma, na)), dtype=np.float32)
    b = np.asfortranarray(rng.uniform(-1, 1, (mb, nb)), dtype=np.float32)
    c0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)), dtype=np.float32)
    c = c0.copy(order="F")
    AB.cblas_sgemm(CM, ta, tb, m, n, k, -0.75, a, ma, b, mb, 0.5, c, m)
    opa = a.astype(np.float64) if ta == 111 else a.astype(np.float64).T
    opb = b.astype(np.float64) if tb == 111 else b.astype(np.float64).T
    ref = -0.75 * (opa @ opb) + 0.5 * c0.astype(np.float64)
    tol = 4 * k * np.finfo(np.float32).eps * (np.abs(opa) @ np.abs(opb)).max()
    assert np.max(np.abs(c - ref)) <= tol


def test_trsm_trmm_golden_cases(gpu, orc, gold):
    for i in range(int(gold["counts"][1])):
        m, n, side, uplo, ta, diag, alpha = gold[f"trsm{i}"]
        m, n, side, uplo, ta, diag = map(int, (m, n, side, uplo, ta, diag))
        a = gold[f"trsm{i}_A"]
        b = np.array(gold[f"trsm{i}_B0"], order="F")
        AB.cblas_dtrsm(CM, side, uplo, ta, diag, m, n, alpha, a, a.shape[0], b, b.shape[0])
        x = gold[f"trsm{i}_X"]
        assert np.max(np.abs(b[:m, :n] - x[:m, :n])) <= 1e-12 * max(m, n), f"trsm case {i}"
        assert orc.gechkgap(b, m, n) == 0
        bm = np.array(gold[f"trsm{i}_B0"], order="F")
        AB.cblas_dtrmm(CM, side, uplo, ta, diag, m, n, alpha, a, a.shape[0], bm, bm.shape[0])
        assert np.max(np.abs(bm[:m, :n] - gold[f"trsm{i}_TB"][:m, :n])) <= 1e-12 * max(m, n), f"trmm {i}"


@pytest.mark.parametrize("side", [141, 142])
@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("ta", [111, 112])
def test_trsm_large_vs_oracle(gpu, orc, side, uplo, ta):
    m, n = (300, 45) if side == 141 else (45, 300)
    na = m if side == 141 else n
    a = orc.gegen(na, na, na, 17)
    orc.trddom(uplo, a, na)
    b0 = orc.gegen(m, n, m, 19)
    b = b0.copy(order="F")
    AB.cblas_dtrsm(CM, side, uplo, ta, 131, m, n, 2.0, a, na, b, m)
    x = orc.dtrsm(side, uplo, ta, 131, m, n, 2.0, a, b0.copy(order="F"))
    assert np.max(np.abs(b - x)) <= 1e-12 * max(m, n) * max(1, np.abs(x).max())


def test_trsm_row_major(gpu, orc):
    m, n = 40, 30
    a = orc.gegen(m, m, m, 3)
    orc.trddom(122, a, m)
    b = orc.uniform((m, n), 4)
    # row-major B (m x n) with ldb = n; A row-major lower
    Ar = np.ascontiguousarray(a)
    Br = np.ascontiguousarray(b)
    AB.cblas_dtrsm(RM, 141, 122, 111, 131, m, n, 1.0, Ar, m, Br, n)
    L = np.tril(a)
    np.testing.assert_allclose(L @ Br, b, rtol=1e-11, atol=1e-11)


def test_syrk_golden_cases(gpu, orc, gold):
    for i in range(int(gold["counts"][2])):
        n, k, uplo, tr, alpha, beta = gold[f"syrk{i}"]
        n, k, uplo, tr = map(int, (n, k, uplo, tr))
        a = gold[f"syrk{i}_A"]
        c = np.array(gold[f"syrk{i}_C0"], order="F")
        AB.cblas_dsyrk(CM, uplo, tr, n, k, alpha, a, a.shape[0], beta, c, c.shape[0])
        ref = gold[f"syrk{i}_C"]
        assert np.max(np.abs(c[:n, :n] - ref[:n, :n])) <= 1e-13 * max(1, k), f"syrk case {i}"
        # the other triangle is untouched
        c0 = gold[f"syrk{i}_C0"]
        mask = np.tril(np.ones((n, n), bool), -1) if uplo == 121 else np.triu(np.ones((n, n), bool), 1)
        assert np.array_equal(c[:n, :n][mask], c0[:n, :n][mask])
        assert orc.gechkgap(c, n, n) == 0
