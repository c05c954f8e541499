"""The multi-GPU entry points of atlas_b200.parallel on one GPU (world size 1:
no collective runs; the GPU kernels do): the column-sharded DGEMM and Ozaki
DGEMM give the product, the batched SPD split solves every problem.  Runs on
more GPUs are not available here; the decomposition and collectives are
covered by tests/test_parallel_host.py on gloo ranks."""
import numpy as np
import pytest

from atlas_b200 import parallel as PAR

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("slices", [0, 8])
def test_sharded_dgemm_one_rank(gpu, slices):
    import torch
    m, n, k = 300, 500, 200
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    A = torch.rand(m, k, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    B = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    C = torch.rand(m, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a_store = A.t().contiguous()
    b_slab = B.t().contiguous()
    c_slab = C.t().contiguous()
    s, w = PAR.sharded_dgemm(a_store, b_slab, c_slab, m, n, k, alpha=0.5, beta=2.0, slices=slices)
    import atlas_b200 as AB
    assert AB.atlb_sync() == 0
    assert (s, w) == (0, n)
    ref = 0.5 * A @ B + 2.0 * C
    err = ((c_slab.t() - ref).abs().max() / ref.abs().max()).item()
    assert err < 1e-14, err


def test_sharded_posv_batched_one_rank(gpu):
    import torch
    rng = np.random.default_rng(4)
    sizes = rng.integers(8, 200, 60).astype(np.int32)
    As, Bs, A0, B0 = [], [], [], []
    for n in sizes:
        G = torch.from_numpy(rng.standard_normal((n, n))).cuda()
        a = G @ G.t() + n * torch.eye(int(n), dtype=torch.float64, device="cuda")
        b = torch.from_numpy(rng.uniform(-1, 1, (4, n))).cuda()   # column-major n x 4
        A0.append(a.clone())
        B0.append(b.clone())
        As.append(a)
        Bs.append(b)
    aptr = [t.data_ptr() for t in As]
    bptr = [t.data_ptr() for t in Bs]
    idx, info = PAR.sharded_posv_batched(sizes, aptr, sizes, bptr, sizes, np.full(len(sizes), 4))
    assert sorted(idx.tolist()) == list(range(len(sizes)))
    assert np.all(info == 0)
    for i in range(len(sizes)):
        x = Bs[i].t()
        r = (A0[i] @ x - B0[i].t()).abs().max().item()
        assert r <= 1e-10 * A0[i].abs().max().item() * max(1.0, x.abs().max().item()), (i, r)


@pytest.mark.parametrize("world", [2, 3, 4])
@pytest.mark.parametrize("slices", [0, 7])
def test_column_slabs_through_the_gpu_kernels(gpu, world, slices):
    """Every rank's slab of a sharded DGEMM, run one after another on this GPU
    through the GEMM each rank would call (DMMA or Ozaki), assembles the full
    product: the slab offsets, widths and leading dimensions are right for
    world sizes the pool cannot give as separate GPUs."""
    import torch
    import atlas_b200 as AB
    m, n, k = 257, 1000, 300
    g = torch.Generator(device="cuda")
    g.manual_seed(11 + world)
    A = torch.rand(m, k, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    B = torch.rand(k, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    C = torch.rand(m, n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    a_store = A.t().contiguous()
    out = C.clone()
    for r, (s, w) in enumerate(PAR.column_slabs(n, world)):
        b_slab = B[:, s:s + w].t().contiguous()
        c_slab = C[:, s:s + w].t().contiguous()
        PAR._default_gemm(111, 111, m, w, k, 0.5, a_store, m, b_slab, k, -1.0, c_slab, m, slices=slices)
        assert AB.atlb_sync() == 0
        out[:, s:s + w] = c_slab.t()
    ref = 0.5 * A @ B - C
    err = ((out - ref).abs().max() / ref.abs().max()).item()
    assert err < (1e-14 if slices == 0 else 1e-12), err
