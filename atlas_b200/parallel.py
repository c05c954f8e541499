"""Multi-GPU work split for the paths that shard: one process per GPU,
torch.distributed (NCCL over NVLink) for the plumbing.

The reference parallelises inside one CPU node: ATL_dtgemm splits C into
blocks among pthreads (src/threads/blas/level3/ATL_tgemm.c:541-628), and a
batch of independent problems is simply divided among threads.  Across GPUs
the same decomposition needs no exchange on the data path:

* DGEMM / split-integer (Ozaki) DGEMM: C is split by column slabs.  A rank
  computes C[:, slab] = alpha * op(A) * op(B)[:, slab] + beta * C[:, slab]
  and needs all of A and only its slab of B and C.  When A lives on one rank
  it is broadcast once (NCCL); nothing else crosses NVLink.  Slab widths are
  multiples of 128 (the GEMM tile) so every rank runs whole tiles.
* Batched solves / GEMMs: the problems are dealt out by work (greedy,
  largest first, onto the least-loaded rank), each rank runs its share in one
  persistent launch.
* One large factorization (getrf / potrf / geqrf) does not shard (its panel
  chain is sequential): `bench.py --gpus N` runs N independent replicas.

Timing across ranks is device time, reduced with MAX (the slowest rank
sets the job's time).  Every TMA load of the kernels these paths run reads
this GPU's own memory into the issuing CTA alone, so they may run on several
GPUs.
"""
import numpy as np

TILE = 128


def column_slabs(n, world, tile=TILE):
    """(start, width) of each rank's column slab of an n-column output:
    contiguous, disjoint, covering [0, n), widths multiples of `tile` except
    possibly the last non-empty one, as equal as whole tiles allow."""
    if world < 1:
        raise ValueError("world must be >= 1")
    ntiles = (n + tile - 1) // tile
    out = []
    t0 = 0
    for r in range(world):
        t1 = t0 + ntiles // world + (1 if r < ntiles % world else 0)
        s, e = min(n, t0 * tile), min(n, t1 * tile)
        out.append((s, e - s))
        t0 = t1
    return out


def split_by_work(work, world):
    """Deal problems out to ranks by work (largest first onto the least-loaded
    rank; ties to the lower rank).  Returns one sorted index array per rank."""
    work = np.asarray(work, dtype=np.float64)
    order = np.argsort(-work, kind="stable")
    load = np.zeros(world)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += work[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def max_over_ranks(value, group=None):
    """MAX of a float over the ranks of the default (or given) process group;
    the value itself when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def _default_gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, slices=0):
    import atlas_b200 as AB
    if slices:
        r = AB.atlb_dgemm_ozaki_dev(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, slices)
    else:
        r = AB.atlb_dgemm_dev(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    if r != 0:
        raise ValueError(f"atlb_dgemm{'_ozaki' if slices else ''}_dev: bad argument {-r}")


def sharded_dgemm(a_store, b_slab, c_slab, m, n, k, alpha=1.0, beta=0.0, src=0, slices=0, group=None,
                  gemm=None):
    """C[:, slab] = alpha * A * B[:, slab] + beta * C[:, slab] (no transposes)
    on this rank, C split by `column_slabs(n, world)`.

    Storage is column-major, held in torch tensors as their transposes:
    a_store is the (k, m) tensor whose memory is the m x k matrix A (lda = m);
    b_slab (w, k) holds this rank's k x w slab of B, c_slab (w, m) its m x w
    slab of C.  A is broadcast from rank `src` (the other ranks' a_store is
    overwritten).  slices > 0 runs the split-integer (Ozaki) GEMM with that
    many slices.  `gemm` replaces the GPU GEMM (tests of the host logic on
    CPU ranks only).  Returns this rank's slab (start, width)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    if world > 1:
        dist.broadcast(a_store, src=src, group=group)
    s, w = column_slabs(n, world)[rank]
    if w > 0 and m > 0:
        (gemm or _default_gemm)(111, 111, m, w, k, alpha, a_store, max(m, 1), b_slab, max(k, 1), beta,
                                c_slab, max(m, 1), slices=slices)
    return s, w


def sharded_posv_batched(n, a_ptrs, lda, b_ptrs, ldb, nrhs, group=None, solve=None):
    """The batched SPD solves of one job split across ranks: every rank gets
    the same problem list (host arrays of sizes, leading dimensions and this
    rank's device pointers -- entries for problems it does not own are not
    read), takes its share by work (n^3/3 + 2 n^2 nrhs, `split_by_work`) and
    solves it in one persistent launch (atlb_dposv_batched).  Returns
    (indices solved here, their info codes).  `solve(idx, ...)` replaces the
    GPU call (tests of the host logic on CPU ranks only)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    n = np.asarray(n, dtype=np.int32)
    nrhs = np.asarray(nrhs, dtype=np.int32)
    work = n.astype(np.float64) ** 3 / 3.0 + 2.0 * n.astype(np.float64) ** 2 * nrhs
    idx = split_by_work(work, world)[rank]
    if solve is not None:
        return idx, solve(idx)
    import atlas_b200 as AB
    cnt = len(idx)
    info = np.zeros(max(cnt, 1), dtype=np.int32)
    if cnt:
        sub = lambda arr, t: np.ascontiguousarray(np.asarray(arr)[idx], dtype=t)
        ap, bp = sub(a_ptrs, np.uint64), sub(b_ptrs, np.uint64)
        r = AB.atlb_dposv_batched(cnt, sub(n, np.int32), ap.ctypes.data, sub(lda, np.int32),
                                  bp.ctypes.data, sub(ldb, np.int32), sub(nrhs, np.int32), info)
        if r != 0:
            raise ValueError(f"atlb_dposv_batched: bad argument {-r}")
    return idx, info[:cnt]
