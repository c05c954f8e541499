"""atlb_dtrsm_dev_noalloc -- the triangular solve for callers that cannot
let the library allocate device memory (graph capture, externally owned
memory pools, fixed budgets) -- must give the results of the regular
atlb_dtrsm_dev, call after call, although its workspace is one fixed array
shared by all calls.  This file is collected last so that a failure here
leaves every other test already run; it also passes alone in a fresh process."""
import pytest

import atlas_b200 as AB

pytestmark = pytest.mark.gpu


def _case(torch, side, m, n, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    na = m if side == 141 else n
    a = torch.rand(na, na, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a = a / na + torch.eye(na, dtype=torch.float64, device="cuda") * 2.0   # well conditioned
    b = torch.rand(n, m, dtype=torch.float64, device="cuda", generator=g) * 2 - 1  # col-major m x n storage
    return a, b, na


@pytest.mark.parametrize("calls", [
    [(141, 122, 111, 131, 700, 90, 1), (142, 121, 112, 132, 50, 1000, 2)],
    [(142, 122, 111, 131, 300, 333, 3), (141, 121, 112, 131, 4096, 8, 4)],
])
def test_noalloc_trsm_matches_trsm_on_consecutive_calls(gpu, calls):
    import torch
    for side, uplo, trans, diag, m, n, seed in calls:
        a, b0, na = _case(torch, side, m, n, seed)
        b_ref = b0.clone()
        b_new = b0.clone()
        assert AB.atlb_dtrsm_dev(side, uplo, trans, diag, m, n, 0.5, a, na, b_ref, m) == 0
        assert AB.atlb_dtrsm_dev_noalloc(side, uplo, trans, diag, m, n, 0.5, a, na, b_new, m) == 0
        AB.atlb_sync()
        # same kernels and workspace layout: the results agree to rounding
        assert torch.allclose(b_new, b_ref, rtol=1e-12, atol=1e-12)
        assert torch.isfinite(b_new).all()


def test_noalloc_trsm_rejects_orders_beyond_its_array(gpu):
    import torch
    m, n = 4097, 2
    a = torch.eye(m, dtype=torch.float64, device="cuda")
    b = torch.ones(n, m, dtype=torch.float64, device="cuda")
    assert AB.atlb_dtrsm_dev_noalloc(141, 122, 111, 131, m, n, 1.0, a, m, b, m) == -5
    assert AB.atlb_dtrsm_dev_noalloc(142, 122, 111, 131, n, m, 1.0, a, m, b.reshape(m, n), n) == -6
    AB.atlb_sync()
    assert torch.all(b == 1.0)
