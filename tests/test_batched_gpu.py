"""Batched uneven-size problems (one persistent launch per batch) against a
per-instance loop of the oracle / numpy: batched Cholesky solve, batched LU
(ipiv identical to the oracle's getrf on each instance) with solve, and the
grouped DGEMM (l3blastst residual per instance)."""
import ctypes

import numpy as np
import pytest

import atlas_b200 as AB
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _ptr_array(ts, ctype=ctypes.c_void_p):
    return (ctype * len(ts))(*[t.data_ptr() for t in ts])


def _int_array(v):
    return np.ascontiguousarray(v, dtype=np.int32)


def test_batched_posv(gpu):
    import torch
    rng = np.random.default_rng(0)
    count = 300
    ns = rng.integers(8, 257, count)
    ns[:3] = [8, 96, 97]          # the size-bucket edges
    nr = 4
    As, Bs, a0s, b0s = [], [], [], []
    for n in ns:
        g = rng.standard_normal((n, n))
        a = g @ g.T + n * np.eye(n)           # A = B B^T + n I
        b = rng.uniform(-1, 1, (n, nr))
        a0s.append(a); b0s.append(b)
        As.append(torch.tensor(np.asfortranarray(a).T.copy(), device="cuda"))   # column-major storage
        Bs.append(torch.tensor(np.asfortranarray(b).T.copy(), device="cuda"))
    info = np.zeros(count, dtype=np.int32)
    r = AB.atlb_dposv_batched(count, _int_array(ns), _ptr_array(As), _int_array(ns), _ptr_array(Bs),
                              _int_array(ns), _int_array([nr] * count), info)
    assert r == 0 and np.all(info == 0)
    for i in range(count):
        x = Bs[i].cpu().numpy().T
        res = np.abs(a0s[i] @ x - b0s[i]).max() / (np.abs(a0s[i]).sum(1).max() * np.abs(x).max())
        assert res < 1e-14, (i, ns[i], res)
        L = np.tril(As[i].cpu().numpy().T)
        np.testing.assert_allclose(L, np.linalg.cholesky(a0s[i]), rtol=1e-10, atol=1e-12)


def test_batched_posv_reports_indefinite(gpu):
    import torch
    ns = np.array([20, 150], dtype=np.int32)
    As, Bs = [], []
    for n in ns:
        a = np.eye(n) * 2.0
        a[n // 2, n // 2] = -1.0
        As.append(torch.tensor(a, device="cuda"))
        Bs.append(torch.ones(1, n, dtype=torch.float64, device="cuda"))
    info = np.zeros(2, dtype=np.int32)
    assert AB.atlb_dposv_batched(2, ns, _ptr_array(As), ns, _ptr_array(Bs), ns, _int_array([1, 1]), info) == 0
    assert list(info) == [n // 2 + 1 for n in ns]


def test_batched_gesv_matches_oracle(gpu, orc):
    import torch
    rng = np.random.default_rng(1)
    count = 120
    ns = rng.integers(8, 257, count)
    ns[:4] = [8, 160, 161, 256]   # shared-memory / global-memory edge
    As, Bs, Ps, a0s, b0s = [], [], [], [], []
    for k, n in enumerate(ns):
        a = O.gegen(int(n), int(n), int(n), 7 + k)[:n, :n].copy(order="F")   # random pivots
        b = rng.uniform(-1, 1, (n, 2))
        a0s.append(a); b0s.append(b)
        As.append(torch.tensor(a.T.copy(), device="cuda"))
        Bs.append(torch.tensor(np.asfortranarray(b).T.copy(), device="cuda"))
        Ps.append(torch.zeros(n, dtype=torch.int32, device="cuda"))
    info = np.zeros(count, dtype=np.int32)
    r = AB.atlb_dgesv_batched(count, _int_array(ns), _ptr_array(As), _int_array(ns), _ptr_array(Ps),
                              _ptr_array(Bs), _int_array(ns), _int_array([2] * count), info)
    assert r == 0 and np.all(info == 0)
    for i in range(count):
        lu, rpiv, _ = orc.dgetrf(a0s[i].copy(order="F"))
        np.testing.assert_array_equal(Ps[i].cpu().numpy(), rpiv)
        assert np.max(np.abs(As[i].cpu().numpy().T - lu)) < 1e-10
        x = Bs[i].cpu().numpy().T
        xt = np.asfortranarray(np.linalg.solve(a0s[i], b0s[i]))   # the oracle reads column-major
        assert orc.resid_slv(a0s[i], np.asfortranarray(x), xt) <= 100


def test_batched_dgemm_uneven(gpu, orc):
    import torch
    rng = np.random.default_rng(2)
    count = 200
    M, N, K = (rng.integers(16, 513, count) for _ in range(3))
    As = [torch.rand(k, m, dtype=torch.float64, device="cuda") * 2 - 1 for m, k in zip(M, K)]   # col-major m x k
    Bs = [torch.rand(n, k, dtype=torch.float64, device="cuda") * 2 - 1 for k, n in zip(K, N)]
    Cs = [torch.rand(n, m, dtype=torch.float64, device="cuda") for m, n in zip(M, N)]
    C0 = [c.clone() for c in Cs]
    r = AB.atlb_dgemm_batched_dev(111, 111, count, _int_array(M), _int_array(N), _int_array(K), 1.5,
                                  _ptr_array(As), _int_array(M), _ptr_array(Bs), _int_array(K), -0.5,
                                  _ptr_array(Cs), _int_array(M))
    assert r == 0
    AB.atlb_sync()
    for i in range(count):
        a = np.asfortranarray(As[i].cpu().numpy().T)
        b = np.asfortranarray(Bs[i].cpu().numpy().T)
        c0 = np.asfortranarray(C0[i].cpu().numpy().T)
        c = np.asfortranarray(Cs[i].cpu().numpy().T)
        assert orc.resid_gemm(111, 111, int(M[i]), int(N[i]), int(K[i]), 1.5, a, b, -0.5, c0, c) < 50


@pytest.mark.parametrize("small,pw", [(96, 32), (128, 16), (64, 64)])
def test_batched_posv_buckets_and_graph_replays(gpu, small, pw):
    """Every size bucket setting of the tuner gives the same solves, and the
    third and later calls of one batch shape (replayed from a CUDA graph) solve
    the new data each call carries."""
    import torch
    old = (AB.atlb_tune_get("batch_posv_small"), AB.atlb_tune_get("batch_posv_pw"))
    AB.atlb_tune_set("batch_posv_small", small)
    AB.atlb_tune_set("batch_posv_pw", pw)
    try:
        rng = np.random.default_rng(small + pw)
        count, nr = 64, 2
        ns = rng.integers(8, 257, count)
        ns[:4] = [small, small + 1, 8, 256]
        for call in range(4):
            As, Bs, a0s, b0s = [], [], [], []
            for n in ns:
                g = rng.standard_normal((n, n))
                a = g @ g.T + n * np.eye(n)
                b = rng.uniform(-1, 1, (n, nr))
                a0s.append(a)
                b0s.append(b)
                As.append(torch.tensor(a, device="cuda"))            # symmetric: either order
                Bs.append(torch.tensor(np.ascontiguousarray(b.T), device="cuda"))
            info = np.zeros(count, dtype=np.int32)
            assert AB.atlb_dposv_batched(count, _int_array(ns), _ptr_array(As), _int_array(ns), _ptr_array(Bs),
                                         _int_array(ns), _int_array([nr] * count), info) == 0
            assert np.all(info == 0)
            for i in range(count):
                x = Bs[i].cpu().numpy().T
                res = np.abs(a0s[i] @ x - b0s[i]).max() / (np.abs(a0s[i]).sum(1).max() * np.abs(x).max())
                assert res < 1e-14, (call, i, ns[i], res)
    finally:
        AB.atlb_tune_set("batch_posv_small", old[0])
        AB.atlb_tune_set("batch_posv_pw", old[1])


def test_batched_getrf_only_matches_oracle(gpu):
    import torch
    rng = np.random.default_rng(21)
    count = 40
    ns = rng.integers(8, 257, count)
    As, Ps, a0s = [], [], []
    for n in ns:
        a = O.lu_matrix(int(n), int(n) + 1)
        a0s.append(a)
        As.append(torch.tensor(np.ascontiguousarray(a.T), device="cuda"))
        Ps.append(torch.zeros(int(n), dtype=torch.int32, device="cuda"))
    info = np.zeros(count, dtype=np.int32)
    for _ in range(3):  # replays from the graph on the later calls
        for i, a in enumerate(a0s):
            As[i].copy_(torch.tensor(np.ascontiguousarray(a.T), device="cuda"))
        assert AB.atlb_dgetrf_batched(count, _int_array(ns), _ptr_array(As), _int_array(ns), _ptr_array(Ps),
                                      info) == 0
        assert np.all(info == 0)
        for i in range(count):
            ref, rpiv, _ = O.dgetrf(a0s[i].copy(order="F"))
            np.testing.assert_array_equal(Ps[i].cpu().numpy(), rpiv)
            assert np.abs(As[i].cpu().numpy().T - ref).max() < 1e-12


def test_batched_getrf_ties_and_zero_columns_match_oracle(gpu):
    """Pivot ties (entries in {-2..2}: many equal |values| per column, the
    first maximum wins) and exactly-zero columns (info = first zero pivot,
    1-based; the factorization completes, as ATL_getf2 does), on sizes that
    cross the 16-column panels of the batched LU."""
    import torch
    ns = [8, 17, 33, 64, 100, 130, 200, 256]
    As, Ps, a0s, zero_col = [], [], [], []
    for k, n in enumerate(ns):
        a = np.asfortranarray(np.round(4.0 * O.gegen(n, n, n, 40 + k)[:n, :n]))
        zc = -1
        if k % 2:          # an exactly-zero column past the first panel
            zc = min(n - 1, 16 + 3 * k)
            a[:, zc] = 0.0
        zero_col.append(zc)
        a0s.append(a)
        As.append(torch.tensor(np.ascontiguousarray(a.T), device="cuda"))
        Ps.append(torch.zeros(n, dtype=torch.int32, device="cuda"))
    info = np.zeros(len(ns), dtype=np.int32)
    assert AB.atlb_dgetrf_batched(len(ns), _int_array(ns), _ptr_array(As), _int_array(ns), _ptr_array(Ps),
                                  info) == 0
    for i, n in enumerate(ns):
        ref, rpiv, rinfo = O.dgetrf(a0s[i].copy(order="F"))
        assert info[i] == rinfo, (n, info[i], rinfo)
        if zero_col[i] >= 0:
            assert rinfo > 0
        np.testing.assert_array_equal(Ps[i].cpu().numpy(), rpiv)
        assert np.abs(As[i].cpu().numpy().T - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
