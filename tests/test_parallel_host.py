"""Host side of the multi-GPU paths, on CPU ranks over gloo (world size 2):
the column-slab split of a sharded DGEMM, the work-balanced split of a
batch, the max-over-ranks timing reduction bench.py uses for its replicas,
and a sharded GEMM end to end with the GPU kernel replaced by numpy (the
broadcast of A, each rank's slab, the gathered result equal to the full
product).  No GPU is used: these check the decomposition and the
collectives, not the kernels (which the -m gpu tests cover on one GPU)."""
import os
import socket

import numpy as np
import pytest

from atlas_b200 import parallel as PAR


def test_column_slabs_cover_disjoint_whole_tiles():
    for n in (1, 127, 128, 129, 1000, 8192):
        for world in (1, 2, 3, 4, 8):
            sl = PAR.column_slabs(n, world)
            assert len(sl) == world
            pos = 0
            for s, w in sl:
                assert s == pos and w >= 0
                pos += w
            assert pos == n
            full = [w for s, w in sl if s + w < n]
            assert all(w % PAR.TILE == 0 for w in full)
            tiles = [(w + PAR.TILE - 1) // PAR.TILE for _, w in sl]
            assert max(tiles) - min(tiles) <= 1


def test_split_by_work_balances_and_covers():
    rng = np.random.default_rng(3)
    sizes = rng.integers(8, 257, 10000)
    work = sizes.astype(float) ** 3
    for world in (1, 2, 4, 8):
        parts = PAR.split_by_work(work, world)
        allidx = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allidx, np.arange(len(sizes)))
        loads = [work[p].sum() for p in parts]
        assert max(loads) - min(loads) <= work.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # max over ranks (bench.py's timing of replicas)
        mx = PAR.max_over_ranks(10.0 + rank)
        # sharded GEMM with a numpy stand-in for the GPU kernel
        m, n, k = 70, 300, 50
        rng = np.random.default_rng(7)
        A = rng.uniform(-1, 1, (m, k))
        B = rng.uniform(-1, 1, (k, n))
        C0 = rng.uniform(-1, 1, (m, n))
        a_store = torch.from_numpy(np.ascontiguousarray(A.T)) if rank == 0 else torch.zeros(k, m, dtype=torch.float64)
        s, w = PAR.column_slabs(n, world)[rank]
        b_slab = torch.from_numpy(np.ascontiguousarray(B[:, s:s + w].T))
        c_slab = torch.from_numpy(np.ascontiguousarray(C0[:, s:s + w].T))
        calls = []

        def np_gemm(ta, tb, mm, nn, kk, alpha, a, lda, b, ldb, beta, c, ldc, slices=0):
            calls.append((mm, nn, kk))
            Am = a.numpy().T[:mm, :kk]
            Bm = b.numpy().T[:kk, :nn]
            Cm = c.numpy().T
            Cm[:mm, :nn] = alpha * Am @ Bm + beta * Cm[:mm, :nn]
            c.copy_(torch.from_numpy(np.ascontiguousarray(Cm.T)))

        s2, w2 = PAR.sharded_dgemm(a_store, b_slab, c_slab, m, n, k, alpha=0.5, beta=2.0, gemm=np_gemm)
        slabs = PAR.column_slabs(n, world)
        wmax = max(wd for _, wd in slabs)
        pad = torch.zeros(wmax, m, dtype=torch.float64)
        pad[:w] = c_slab
        gathered = [torch.zeros(wmax, m, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, pad)   # gloo gathers equal sizes: slabs padded to the widest
        C = np.concatenate([gathered[r][:slabs[r][1]].numpy().T for r in range(world)], axis=1)
        err = float(np.max(np.abs(C - (0.5 * A @ B + 2.0 * C0))))
        a_ok = bool(np.array_equal(a_store.numpy().T, A))
        q.put((rank, mx, (s2, w2) == (s, w), err, a_ok, calls))
    except BaseException as e:  # noqa: BLE001 -- reported to the parent, which fails the test
        q.put((rank, "error", repr(e), None, None, None))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sharded_gemm_and_timing():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, slab_ok, err, a_ok, calls in res:
        assert mx != "error", f"rank {rank}: {slab_ok}"
        assert mx == 11.0
        assert slab_ok
        assert a_ok, f"rank {rank} did not receive A"
        assert err < 1e-12, err
        assert len(calls) == 1 and calls[0][0] == 70 and calls[0][2] == 50


def _bench_worker(rank, world, port, q):
    import sys
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        import bench
        q.put((rank, bench.replica_throughput(10.0 + 2.0 * rank, world)))
    except BaseException as e:  # noqa: BLE001
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_bench_replica_throughput_two_gloo_ranks():
    """bench.py --gpus N: N replicas, value = N solves / slowest rank's time."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        value, ms = res[rank]
        assert ms == 12.0
        assert abs(value - 2 * 1000.0 / 12.0) < 1e-9


def _posv_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(11)
        sizes = rng.integers(8, 257, 500)
        solved = []

        def fake_solve(idx):
            solved.extend(int(i) for i in idx)
            return np.zeros(len(idx), dtype=np.int32)

        idx, info = PAR.sharded_posv_batched(sizes, [0] * 500, sizes, [0] * 500, sizes, [4] * 500,
                                             solve=fake_solve)
        q.put((rank, sorted(solved), float((sizes[idx].astype(float) ** 3).sum())))
    except BaseException as e:  # noqa: BLE001
        q.put((rank, repr(e), None))
    finally:
        dist.destroy_process_group()


def test_batched_split_two_gloo_ranks():
    """Every problem of the batch is solved by exactly one rank, loads balanced."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_posv_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r[0], r[1:]) for r in (q.get(timeout=180) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    both = res[0][0] + res[1][0]
    assert sorted(both) == list(range(500))
    loads = [res[0][1], res[1][1]]
    assert abs(loads[0] - loads[1]) <= 256 ** 3
