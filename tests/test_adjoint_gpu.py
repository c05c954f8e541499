"""Adjoints of potrf/potrs and getrf/getrs (library kernels), wrapped in a
torch.autograd.Function here in the test harness only, checked against the
closed-form gradients and against central finite differences (step 1e-6,
random symmetric directions) of the same loss evaluated with the library's
forward routines."""
import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LOWER, NOTRANS = 122, 111


def _chol(torch, A):
    """Column-major L with A = L L^T (A symmetric, so storage order is moot)."""
    n = A.shape[0]
    L = A.clone()
    info = torch.zeros(1, dtype=torch.int32, device=A.device)
    assert AB.atlb_dpotrf_dev(LOWER, n, L, n, info) == 0
    AB.atlb_sync()
    assert int(info.item()) == 0
    return L  # storage: row-major view of the column-major factor


def gauss_loss_forward(torch, A, y):
    """2 sum log diag(chol(A)) + y^T A^-1 y with the library's potrf / potrs."""
    n = A.shape[0]
    L = _chol(torch, A)
    x = y.clone()
    assert AB.atlb_dpotrs_dev(LOWER, n, 1, L, n, x, n) == 0
    AB.atlb_sync()
    Lc = L.T  # logical column-major factor
    return 2.0 * torch.log(torch.diagonal(Lc)).sum() + torch.dot(y, x), L, x


def make_gauss_fn(torch):
    class GaussLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, A, y):
            val, L, x = gauss_loss_forward(torch, A, y)
            ctx.save_for_backward(L, x, y)
            return val

        @staticmethod
        def backward(ctx, g):
            L, x, y = ctx.saved_tensors
            n = L.shape[0]
            Lc = L.T.contiguous()                       # logical factor, row-major
            Lbar_c = torch.diag(2.0 / torch.diagonal(Lc)) * g   # d(2 sum log L_ii)/dL
            Lbar = Lbar_c.T.contiguous()                # column-major storage
            Abar = torch.zeros_like(L)
            assert AB.atlb_dpotrf_adjoint_dev(n, L, n, Lbar, n, Abar, n) == 0
            Bbar = torch.empty_like(y)
            xbar = (g * y).contiguous()
            assert AB.atlb_dpotrs_adjoint_dev(n, 1, L, n, x, n, xbar, n, Bbar, n, Abar, n) == 0
            AB.atlb_sync()
            return Abar.T.contiguous(), None            # symmetric anyway
    return GaussLoss


@pytest.mark.parametrize("n", [200, 700])
def test_potrf_potrs_adjoint(gpu, n):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(n)
    B = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    A = (B @ B.T / n + torch.eye(n, dtype=torch.float64, device="cuda")).requires_grad_(True)
    y = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    loss = make_gauss_fn(torch).apply(A, y)
    loss.backward()
    grad = A.grad
    Ad = A.detach()
    Ainv = torch.linalg.inv(Ad)
    a = Ainv @ y
    closed = Ainv - torch.outer(a, a)
    assert torch.allclose(grad, closed, rtol=1e-9, atol=1e-11 * closed.abs().max().item())
    # central finite differences on random symmetric directions
    h = 1e-6
    for k in range(16):
        E = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        E = (E + E.T) / 2
        E /= E.norm()
        fp = gauss_loss_forward(torch, Ad + h * E, y)[0].item()
        fm = gauss_loss_forward(torch, Ad - h * E, y)[0].item()
        fd = (fp - fm) / (2 * h)
        an = torch.sum(grad * E).item()
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (k, fd, an)


def _ptrs(np_, ts):
    return np_.array([t.data_ptr() for t in ts], dtype=np_.uint64)


def test_potrf_potrs_adjoint_batched_512x128(gpu):
    """The Gaussian-likelihood loss of 512 systems at N = 128, its gradient in
    two one-launch batched adjoints (potrf, then potrs) through the C ABI,
    against the closed form A^-1 - a a^T of every system."""
    import torch
    count, n = 512, 128
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    As, Ls, Ys, Xs = [], [], [], []
    for _ in range(count):
        B = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        A = B @ B.T / n + torch.eye(n, dtype=torch.float64, device="cuda")
        As.append(A)
        Ls.append(A.clone())
        y = torch.rand(1, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        Ys.append(y)
        Xs.append(y.clone())
    nv = np.full(count, n, np.int32)
    info = np.zeros(count, np.int32)
    # forward: L (lower) and x = A^-1 y for every system in one launch
    assert AB.atlb_dposv_batched(count, nv, _ptrs(np, Ls), nv, _ptrs(np, Xs), nv, np.ones(count, np.int32),
                                 info) == 0
    assert np.all(info == 0)
    Lbars, Abars, Bbars = [], [], []
    for L in Ls:
        Lc = L.T   # logical column-major factor
        Lbars.append(torch.diag(2.0 / torch.diagonal(Lc)).T.contiguous())
        Abars.append(torch.zeros(n, n, dtype=torch.float64, device="cuda"))
        Bbars.append(torch.zeros(1, n, dtype=torch.float64, device="cuda"))
    assert AB.atlb_dpotrf_adjoint_batched_dev(count, nv, _ptrs(np, Ls), nv, _ptrs(np, Lbars), nv,
                                              _ptrs(np, Abars), nv) == 0
    assert AB.atlb_dpotrs_adjoint_batched_dev(count, nv, np.ones(count, np.int32), _ptrs(np, Ls), nv,
                                              _ptrs(np, Xs), nv, _ptrs(np, Ys), nv, _ptrs(np, Bbars), nv,
                                              _ptrs(np, Abars), nv) == 0
    assert AB.atlb_sync() == 0
    worst = 0.0
    for k in range(count):
        Ainv = torch.linalg.inv(As[k])
        a = Ainv @ Ys[k][0]
        closed = Ainv - torch.outer(a, a)
        worst = max(worst, ((Abars[k].T - closed).abs().max() / closed.abs().max()).item())
        if k < 8:  # the same numbers as the unbatched kernels
            Ab1 = torch.zeros(n, n, dtype=torch.float64, device="cuda")
            Bb1 = torch.zeros(1, n, dtype=torch.float64, device="cuda")
            assert AB.atlb_dpotrf_adjoint_dev(n, Ls[k], n, Lbars[k], n, Ab1, n) == 0
            assert AB.atlb_dpotrs_adjoint_dev(n, 1, Ls[k], n, Xs[k], n, Ys[k], n, Bb1, n, Ab1, n) == 0
            assert AB.atlb_sync() == 0
            assert torch.allclose(Ab1, Abars[k], rtol=1e-10, atol=1e-12)
    assert worst < 1e-10, worst


def test_potrf_potrs_adjoint_4096_fd_64_directions(gpu):
    """The benchmark configuration: N = 4096, A = B B^T / N + I, y uniform[-1,1];
    the gradient against the closed form and central finite differences
    (step 1e-6) on 64 random symmetric directions."""
    import torch
    n = 4096
    g = torch.Generator(device="cuda")
    g.manual_seed(4096)
    B = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    A = (B @ B.T / n + torch.eye(n, dtype=torch.float64, device="cuda")).requires_grad_(True)
    del B
    y = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    make_gauss_fn(torch).apply(A, y).backward()
    grad = A.grad
    Ad = A.detach()
    Ainv = torch.linalg.inv(Ad)
    a = Ainv @ y
    closed = Ainv - torch.outer(a, a)
    assert ((grad - closed).abs().max() / closed.abs().max()).item() < 1e-9
    del Ainv, closed
    h = 1e-6
    for k in range(64):
        E = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        E = (E + E.T) / 2
        E /= E.norm()
        fp = gauss_loss_forward(torch, Ad + h * E, y)[0].item()
        fm = gauss_loss_forward(torch, Ad - h * E, y)[0].item()
        an = torch.sum(grad * E).item()
        assert abs((fp - fm) / (2 * h) - an) <= 1e-5 * max(1.0, abs(an)), (k, (fp - fm) / (2 * h), an)


def _lu(torch, Acol, n):
    LU = Acol.clone()
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert AB.atlb_dgetrf_dev(n, n, LU, n, ipiv, info) == 0
    AB.atlb_sync()
    return LU, ipiv


@pytest.mark.parametrize("n", [300, 4096])
def test_getrs_adjoint_closed_form_and_fd(gpu, n):
    """L(A) = c^T A^-1 b (A = G/sqrt(n) + 4I; n = 4096 is the benchmark
    configuration): the getrs adjoint against the closed form -A^-T c (A^-1 b)^T
    and central finite differences."""
    import torch
    a0 = O.lu_matrix(n, 21)
    Acol = torch.tensor(np.ascontiguousarray(a0.T), device="cuda")  # storage of column-major a0
    rng = np.random.default_rng(3)
    b = torch.tensor(rng.uniform(-1, 1, n), device="cuda")
    c = torch.tensor(rng.uniform(-1, 1, n), device="cuda")

    def loss(Ac):
        LU, ipiv = _lu(torch, Ac, n)
        x = b.clone()
        assert AB.atlb_dgetrs_dev(NOTRANS, n, 1, LU, n, ipiv, x, n) == 0
        AB.atlb_sync()
        return torch.dot(c, x).item(), LU, ipiv, x

    val, LU, ipiv, x = loss(Acol)
    Abar = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    Bbar = torch.empty(n, dtype=torch.float64, device="cuda")
    assert AB.atlb_dgetrs_adjoint_dev(n, 1, LU, n, ipiv, x, n, c, n, Bbar, n, Abar, n) == 0
    AB.atlb_sync()
    A = torch.tensor(a0, device="cuda")
    closed = -torch.outer(torch.linalg.solve(A.T, c), torch.linalg.solve(A, b))   # -A^-T c (A^-1 b)^T
    grad = Abar.T                                               # logical column-major
    assert torch.allclose(grad, closed, rtol=1e-10, atol=1e-13)
    h = 1e-6
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    for k in range(8):
        E = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        E /= E.norm()
        fp = loss(Acol + h * E.T.contiguous())[0]
        fm = loss(Acol - h * E.T.contiguous())[0]
        assert abs((fp - fm) / (2 * h) - torch.sum(grad * E).item()) <= 1e-6 * max(1.0, abs(val))


def test_getrf_adjoint_fd(gpu):
    """Adjoint of the factors: f(A) = <W_L, L(A)> + <W_U, U(A)>."""
    import torch
    n = 150
    a0 = O.lu_matrix(n, 4)
    Acol = torch.tensor(a0.T.copy(), device="cuda")
    rng = np.random.default_rng(8)
    WL = torch.tensor(np.tril(rng.standard_normal((n, n)), -1), device="cuda")   # logical
    WU = torch.tensor(np.triu(rng.standard_normal((n, n))), device="cuda")

    def f(Ac):
        LU, ipiv = _lu(torch, Ac, n)
        M = LU.T  # logical LU
        return (torch.sum(WL * torch.tril(M, -1)) + torch.sum(WU * torch.triu(M))).item(), LU, ipiv

    _, LU, ipiv = f(Acol)
    Abar = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    assert AB.atlb_dgetrf_adjoint_dev(n, LU, n, ipiv, WL.T.contiguous(), n, WU.T.contiguous(), n, Abar, n) == 0
    AB.atlb_sync()
    grad = Abar.T
    h = 1e-6
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    for k in range(8):
        E = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        E /= E.norm()
        fp = f(Acol + h * E.T.contiguous())[0]
        fm = f(Acol - h * E.T.contiguous())[0]
        an = torch.sum(grad * E).item()
        assert abs((fp - fm) / (2 * h) - an) <= 1e-5 * max(1.0, abs(an)), (k, an)
