"""atlb_dtrsm_dev_noalloc -- the triangular solve for callers that cannot
let the library allocate device memory (applications whose device memory
belongs to their own pool or framework allocator, fixed memory budgets) --
must solve the same systems as the regular atlb_dtrsm_dev, call after call,
although its workspace is one fixed array shared by all calls.  Each result
is also checked against an FP64 triangular solve on the host (torch on the
CPU), which shares no code with the library.  The no-allocation call comes
first in every case, so its workspace is never one that an earlier regular
call had already sized.  This file is collected last so that a failure here
leaves every other test already run; it also passes alone in a fresh process."""
import threading

import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu

LEFT, RIGHT, UPPER, LOWER, NOTRANS, TRANS, NONUNIT, UNIT = 141, 142, 121, 122, 111, 112, 131, 132


def _case(torch, side, m, n, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    na = m if side == LEFT else n
    a = torch.rand(na, na, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a = a / na + torch.eye(na, dtype=torch.float64, device="cuda") * 2.0   # well conditioned
    b = torch.rand(n, m, dtype=torch.float64, device="cuda", generator=g) * 2 - 1  # col-major m x n storage
    return a, b, na


def _host_solve(torch, side, uplo, trans, diag, alpha, a_cm, b_cm):
    """X with op(A) X = alpha B (Left) or X op(A) = alpha B (Right), FP64 on
    the CPU.  a_cm / b_cm are the column-major buffers viewed as C-ordered
    tensors, i.e. their transposes."""
    A = a_cm.cpu().T.contiguous()
    B = b_cm.cpu().T.contiguous() * alpha
    T = torch.tril(A) if uplo == LOWER else torch.triu(A)
    if diag == UNIT:
        T = T - torch.diag(torch.diag(T)) + torch.eye(T.shape[0], dtype=T.dtype)
    if trans != NOTRANS:
        T = T.T.contiguous()
    up = bool(torch.equal(T, torch.triu(T)))
    if side == LEFT:
        X = torch.linalg.solve_triangular(T, B, upper=up, left=True)
    else:
        X = torch.linalg.solve_triangular(T, B, upper=up, left=False)
    return X.T.contiguous()  # back to the column-major buffer's view


def _check(torch, side, uplo, trans, diag, m, n, seed):
    a, b0, na = _case(torch, side, m, n, seed)
    b_new = b0.clone()
    b_ref = b0.clone()
    assert AB.atlb_dtrsm_dev_noalloc(side, uplo, trans, diag, m, n, 0.5, a, na, b_new, m) == 0
    assert AB.atlb_dtrsm_dev(side, uplo, trans, diag, m, n, 0.5, a, na, b_ref, m) == 0
    assert AB.atlb_sync() == 0
    assert torch.isfinite(b_new).all()
    # same kernels and workspace layout as the regular solve: agreement to rounding
    assert torch.allclose(b_new, b_ref, rtol=1e-12, atol=1e-12)
    # an independent FP64 solve (the triangle is diagonally dominant: cond ~ 1)
    x = _host_solve(torch, side, uplo, trans, diag, 0.5, a, b0)
    err = (b_new.cpu() - x).abs().max().item() / max(x.abs().max().item(), 1e-300)
    assert err < 1e-12, err


@pytest.mark.parametrize("calls", [
    [(LEFT, LOWER, NOTRANS, NONUNIT, 700, 90, 1), (RIGHT, UPPER, TRANS, UNIT, 50, 1000, 2)],
    [(RIGHT, LOWER, NOTRANS, NONUNIT, 300, 333, 3), (LEFT, UPPER, TRANS, NONUNIT, 4096, 8, 4)],
])
def test_noalloc_trsm_matches_trsm_on_consecutive_calls(gpu, calls):
    import torch
    for side, uplo, trans, diag, m, n, seed in calls:
        _check(torch, side, uplo, trans, diag, m, n, seed)


def test_noalloc_trsm_from_a_new_host_thread(gpu):
    """A host thread that never touched the GPU gets the library's stream and
    the array's address on the library's device."""
    import torch
    errors = []

    def work():
        try:
            _check(torch, LEFT, UPPER, NOTRANS, NONUNIT, 257, 31, 5)
            _check(torch, LEFT, LOWER, TRANS, UNIT, 129, 7, 6)
        except BaseException as e:  # noqa: BLE001 -- re-raised in the main thread
            errors.append(e)

    t = threading.Thread(target=work)
    t.start()
    t.join()
    if errors:
        raise errors[0]


def test_noalloc_trsm_rejects_orders_beyond_its_array(gpu):
    import torch
    m, n = 4097, 2
    a = torch.eye(m, dtype=torch.float64, device="cuda")
    b = torch.ones(n, m, dtype=torch.float64, device="cuda")
    assert AB.atlb_dtrsm_dev_noalloc(LEFT, LOWER, NOTRANS, NONUNIT, m, n, 1.0, a, m, b, m) == -5
    assert AB.atlb_dtrsm_dev_noalloc(RIGHT, LOWER, NOTRANS, NONUNIT, n, m, 1.0, a, m, b.reshape(m, n), n) == -6
    assert AB.atlb_sync() == 0
    assert torch.all(b == 1.0)
