"""Orders past the limits of the one-launch kernels' fast paths:

* getrs with one right-hand side at n = 20000: the one-launch triangular
  solve then has more 128-row blocks (157) than the GPU holds at once, so
  blocks whose ticket comes later start only when earlier ones finish (the
  tickets keep every wait on a block that is already running);
* getrf and the mixed solver at n = 9000: more rows than one cluster of the
  fused leaf panel holds (16 x 512), so the first blocks go through the
  recursive panel path and the later ones through the fused kernel;
* getrf of a 30000 x 512 matrix: pivot rows up to ~30000 rows below their
  block, farther than the sequential interchange plan can track (24576 rows);
  getrf's pivots take the parallel plan, which keeps only the rows a chunk of
  interchanges touches.

References are computed on the GPU with torch (FP64) and the checks are the
tester-style normwise residuals (bin/lutst.c, bin/slvtst.c: pass <= 100)."""
import numpy as np
import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu

NOTRANS = 111


def _colmajor(t):
    """A row-major torch matrix's column-major storage (a contiguous transpose)."""
    return t.t().contiguous()


def test_getrs_one_rhs_more_blocks_than_resident(gpu):
    import torch
    n = 20000
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    f64 = torch.float64
    L = torch.tril(torch.rand(n, n, dtype=f64, device="cuda", generator=g) * 2 - 1, -1) / n ** 0.5
    L += torch.eye(n, dtype=f64, device="cuda")
    U = torch.triu(torch.rand(n, n, dtype=f64, device="cuda", generator=g) * 2 - 1) / n ** 0.5
    U += torch.diag(torch.rand(n, dtype=f64, device="cuda", generator=g) + 1)
    lu = _colmajor(torch.tril(L, -1) + U)
    ipiv = torch.arange(n, dtype=torch.int32, device="cuda")
    b = torch.rand(n, 1, dtype=f64, device="cuda", generator=g) * 2 - 1
    x = b.clone()
    assert AB.atlb_dgetrs_dev(NOTRANS, n, 1, lu, n, ipiv, x, n) == 0
    AB.atlb_sync()
    y = torch.linalg.solve_triangular(L, b, upper=False, unitriangular=True)
    ref = torch.linalg.solve_triangular(U, y, upper=True)
    err = ((x - ref).abs().max() / ref.abs().max()).item()
    assert err < 1e-12, err


def test_getrf_rows_beyond_one_cluster(gpu):
    import torch
    n = 9000
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    a = torch.rand(n, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    da = _colmajor(a)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert AB.atlb_dgetrf_dev(n, n, da, n, ipiv, info) == 0
    AB.atlb_sync()
    assert int(info.item()) == 0
    f = da.t()                                   # row-major view of the packed factors
    L = torch.tril(f, -1) + torch.eye(n, dtype=torch.float64, device="cuda")
    U = torch.triu(f)
    piv = ipiv.cpu().numpy()                     # the interchanges (0-based) replayed on A's rows
    perm = np.arange(n)
    for k in range(n):
        p = piv[k]
        if p != k:
            perm[k], perm[p] = perm[p], perm[k]
    pa = a[torch.as_tensor(perm, device="cuda")]
    resid = ((pa - L @ U).abs().sum(0).max() / (a.abs().sum(0).max() * n * 2.0 ** -52)).item()
    assert resid <= 100.0, resid
    assert (ipiv.cpu().numpy() >= np.arange(n)).all()   # pivots come from the rows below


def test_mixed_dgesv_rows_beyond_one_cluster(gpu):
    import torch
    n = 9000
    g = torch.Generator(device="cuda")
    g.manual_seed(13)
    a = (torch.rand(n, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1) / n ** 0.5
    a += 2.0 * torch.eye(n, dtype=torch.float64, device="cuda")
    da = _colmajor(a)
    b = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    x = torch.empty_like(b)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    it = np.zeros(1, dtype=np.int32)
    assert AB.atlb_dsgesv_ex(n, 1, da, n, ipiv, b, n, x, n, 3, 0, it) == 0
    AB.atlb_sync()
    assert it[0] >= 0, it[0]                     # refined in mixed precision, no FP64 fallback
    r = b - a @ x
    berr = (r.abs().max() / (a.abs().sum(1).max() * x.abs().max() + b.abs().max())).item()
    assert berr <= n * 2.0 ** -53, berr


def test_getrf_tall_pivots_beyond_plan_span(gpu):
    import torch
    m, n = 30000, 512
    g = torch.Generator(device="cuda")
    g.manual_seed(14)
    a = torch.rand(m, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    da = _colmajor(a)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert AB.atlb_dgetrf_dev(m, n, da, m, ipiv, info) == 0
    AB.atlb_sync()
    assert int(info.item()) == 0
    piv = ipiv.cpu().numpy()
    assert (piv >= np.arange(n)).all() and piv.max() >= 256 + 24576   # some pivots lie beyond a plan's span
    f = da.t()                                   # row-major view (m x n) of the packed factors
    L = torch.tril(f, -1) + torch.eye(m, n, dtype=torch.float64, device="cuda")
    U = torch.triu(f[:n])
    perm = np.arange(m)
    for k in range(n):
        p = piv[k]
        if p != k:
            perm[k], perm[p] = perm[p], perm[k]
    pa = a[torch.as_tensor(perm, device="cuda")]
    resid = ((pa - L @ U).abs().sum(0).max() / (a.abs().sum(0).max() * m * 2.0 ** -52)).item()
    assert resid <= 100.0, resid
