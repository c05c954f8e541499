"""The tcgen05 tensor-core GEMMs (TF32 and BF16 operands, FP32 accumulation)
against an FP64 product of the same rounded operands: the only differences
allowed are FP32 accumulation errors, bounded by K * 2^-23 * sum|a||b|."""
import numpy as np
import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu


def _round(x, prec):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32))
    if prec == 2:
        return t.to(torch.bfloat16).to(torch.float64).numpy()
    # TF32: round to nearest (ties away) at 10 mantissa bits
    u = t.view(torch.int32).numpy().astype(np.int64) & 0xFFFFFFFF
    u = (u + 0x1000) & 0xFFFFE000
    return np.frombuffer(u.astype(np.uint32).tobytes(), dtype=np.float32).reshape(x.shape).astype(np.float64)


@pytest.mark.parametrize("prec", [1, 2, 3])
@pytest.mark.parametrize("ta,tb", [(111, 111), (111, 112), (112, 111), (112, 112)])
@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (300, 200, 517), (1000, 257, 96), (77, 1030, 33)])
def test_tc_sgemm(gpu, orc, prec, ta, tb, m, n, k):
    import torch
    rng = np.random.default_rng(m * 7 + n + k + prec)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == 111 else (k, m)).astype(np.float32))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == 111 else (n, k)).astype(np.float32))
    C0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(np.float32))
    dA = torch.from_numpy(A.T.copy()).cuda()   # torch row-major of A^T == column-major A
    dB = torch.from_numpy(B.T.copy()).cuda()
    dC = torch.from_numpy(C0.T.copy()).cuda()
    lda, ldb = A.shape[0], B.shape[0]
    assert AB.atlb_sgemm_tc_dev(prec, ta, tb, m, n, k, 1.5, dA, lda, dB, ldb, -0.5, dC, m) == 0
    AB.atlb_sync()
    C = dC.cpu().numpy().T
    if prec == 3:   # split TF32: FP32-accurate products of the FP32 operands
        opA = (A if ta == 111 else A.T).astype(np.float64)
        opB = (B if tb == 111 else B.T).astype(np.float64)
    else:
        opA = _round(A, prec) if ta == 111 else _round(A, prec).T
        opB = _round(B, prec) if tb == 111 else _round(B, prec).T
    ref = 1.5 * (opA @ opB) - 0.5 * C0.astype(np.float64)
    bound = 1.5 * k * 2.0 ** -22 * (np.abs(opA) @ np.abs(opB)) + 2.0 ** -22 * np.abs(ref) + 1e-6
    if prec == 3:   # plus the dropped lo*lo term and the TF32 rounding of the low parts
        bound = bound + 1.5 * 2.0 ** -19 * (np.abs(opA) @ np.abs(opB))
    assert np.all(np.abs(C - ref) <= bound), np.max(np.abs(C - ref) / bound)


def test_tc_sgemm_lower_triangle_only(gpu):
    import torch
    n, k = 300, 128
    A = torch.rand(k, n, device="cuda") * 2 - 1      # storage of column-major n x k
    C = torch.full((n, n), 7.0, device="cuda")
    lib = AB.lib()
    # through the factorization path the tri mask is used by SYRK; here via the dev GEMM
    assert AB.atlb_sgemm_tc_dev(1, 111, 112, n, n, k, 1.0, A, n, A, n, 0.0, C, n) == 0
    AB.atlb_sync()
    assert torch.all(torch.isfinite(C))
