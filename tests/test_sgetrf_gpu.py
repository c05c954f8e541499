"""The FP32 LU with partial pivoting inside the mixed-precision solvers,
through the C ABI (atlb_sgetrf_dev): ipiv is a valid interchange sequence,
P A = L U to FP32 rounding (the lutst residual with eps = 2^-23), element
growth stays modest, |L| <= 1, exact zero columns are reported in info, and
single-panel, block and multi-block shapes (rows up to one cluster's 16 x 512)
all hold; the mixed solver built on it converges at N = 8192."""
import numpy as np
import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu
EPS32 = 2.0 ** -23


def _perm(ipiv, m):
    p = np.arange(m)
    for j, r in enumerate(ipiv):
        p[j], p[r] = p[r], p[j]
    return p


def _factor(torch, a, prec):
    """a: logical m x n FP32 (torch, cuda).  Returns (LU logical, ipiv, info)."""
    m, n = a.shape
    buf = a.t().contiguous()                    # column-major storage
    ipiv = torch.zeros(min(m, n), dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert AB.atlb_sgetrf_dev(m, n, buf, m, ipiv, info, prec) == 0
    assert AB.atlb_sync() == 0
    return buf.t(), ipiv.cpu().numpy(), int(info.item())


def _check(torch, a, prec, growth_max=200.0):
    m, n = a.shape
    lu, ipiv, info = _factor(torch, a, prec)
    assert info == 0
    k = min(m, n)
    assert np.all((ipiv >= np.arange(k)) & (ipiv < m)), "ipiv is not an interchange sequence"
    p = torch.from_numpy(_perm(ipiv, m)).cuda()
    L = torch.tril(lu[:, :k].double(), -1)
    L[:k, :k] += torch.eye(k, dtype=torch.float64, device="cuda")
    U = torch.triu(lu[:k, :].double())
    A = a.double()
    r = (A[p] - L @ U).abs().sum(dim=0).max().item() / (A.abs().sum(dim=0).max().item() * EPS32 * k)
    assert r <= 100.0, r
    growth = U.abs().max().item() / A.abs().max().item()
    assert growth <= growth_max, growth
    assert L.abs().max().item() <= 1.0 + 1e-6      # partial pivoting: |multipliers| <= 1


def _kappa(torch, n, kappa, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    q1, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    q2, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    s = torch.logspace(0, -np.log10(kappa), n, dtype=torch.float64, device="cuda")
    return ((q1 * s) @ q2.t()).float()


@pytest.mark.parametrize("m,n", [(40, 32), (700, 32), (8192, 32), (5000, 17), (8192, 256), (3000, 200)])
def test_sgetrf_panels_and_blocks(gpu, m, n):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(m + n)
    a = torch.rand(m, n, device="cuda", generator=g) * 2 - 1
    _check(torch, a, 0)


@pytest.mark.parametrize("n", [100, 513, 1000, 2048])
@pytest.mark.parametrize("prec", [0, 3])
def test_sgetrf_square_uniform(gpu, n, prec):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(n * 7 + prec)
    a = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
    _check(torch, a, prec)


def test_sgetrf_benchmark_matrix_8192(gpu):
    import torch
    _check(torch, _kappa(torch, 8192, 1e2, 3), 3)


def test_sgetrf_zero_column_info(gpu):
    import torch
    n = 600
    g = torch.Generator(device="cuda")
    g.manual_seed(44)
    a = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
    a[:, 77] = 0.0
    _, ipiv, info = _factor(torch, a, 0)
    assert info == 78
    assert np.all((ipiv >= np.arange(n)) & (ipiv < n))


def test_mixed_dsgesv_8192_converges(gpu):
    import torch
    n = 8192
    A = _kappa(torch, n, 1e2, 5).double()
    g = torch.Generator(device="cuda")
    g.manual_seed(6)
    b = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    acol = A.t().contiguous()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsgesv(n, 1, acol, n, ipiv, b, n, x, n, AB.PREC_TF32X3, it) == 0
    assert 0 <= it[0] <= 4, it[0]
    r = (b - A @ x).abs().max().item()
    bwd = r / (A.abs().sum(dim=1).max().item() * x.abs().max().item() + b.abs().max().item())
    assert bwd <= n * 2.0 ** -53, bwd
