"""Empirical search for the drivers' tunable parameters, in the spirit of
ATLAS's install-time tuning (tune/blas/gemm/gmmsearch.c): each parameter's
candidates are timed on this GPU with the others held at their current best
(one coordinate-descent pass), and the winners are written to tuning.conf
beside the library, which reads it on first use.

    python -m atlas_b200.tune [--n 8192] [--out PATH]

Parameters (see atlas_b200/csrc/tuning.cu): getrf_nb, lookahead,
lookahead_reserve_sms, potrf_nb, dgemm_group, dgemm_splitk, sgetrf_nb,
mixed_tc_min_work_log2.
"""
import argparse
import os
import time

import numpy as np

import atlas_b200 as AB


def _timer(torch, stream, fn, reps):
    """Median of `reps` individually timed calls (after one untimed call)."""
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return sorted(times)[len(times) // 2]


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=8192, help="order of the factorization benchmarks")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(AB.LIB_PATH)), "tuning.conf"))
    args = ap.parse_args()

    import torch
    os.environ.setdefault("ATLAS_B200_TUNE_FILE", "none")  # search from the built-in defaults
    AB.lib()
    assert AB.atlb_init(0) == 0
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    AB.atlb_set_stream(stream.cuda_stream)
    dev = torch.device("cuda")
    f64 = torch.float64
    n = args.n
    g = torch.Generator(device=dev)
    g.manual_seed(17)

    a_lu = torch.randn(n, n, dtype=f64, device=dev, generator=g) / n ** 0.5
    gm = torch.randn(n, n, dtype=f64, device=dev, generator=g)
    a_spd = gm @ gm.T / n + torch.eye(n, dtype=f64, device=dev)
    del gm
    work = torch.empty_like(a_lu)
    ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def getrf():
        work.copy_(a_lu)
        AB.atlb_dgetrf_dev(n, n, work, n, ipiv, info)

    def potrf():
        work.copy_(a_spd)
        AB.atlb_dpotrf_dev(122, n, work, n, info)

    m = 8192
    ga = torch.rand(m, m, dtype=f64, device=dev, generator=g)
    gb = torch.rand(m, m, dtype=f64, device=dev, generator=g)
    gc = torch.zeros(m, m, dtype=f64, device=dev)

    def dgemm_big():
        AB.atlb_dgemm_dev(111, 111, m, m, m, 1.0, ga, m, gb, m, 0.0, gc, m)

    small = [(256, 8192, 256), (8192, 256, 256), (512, 512, 4096), (4096, 224, 32), (128, 8192, 128)]

    def dgemm_small():
        for (mm, nn, kk) in small:
            AB.atlb_dgemm_dev(111, 111, mm, nn, kk, -1.0, ga, m, gb, m, 1.0, gc, m)

    x = torch.empty(n, dtype=f64, device=dev)
    b = torch.rand(n, dtype=f64, device=dev, generator=g) * 2 - 1
    it = np.zeros(1, dtype=np.int32)
    # the mixed solvers are timed on the matrix class of the dgesv benchmark:
    # Q1 diag(s) Q2^T, Q from QR of Gaussian matrices, s geometric, cond 1e2
    q1, _ = torch.linalg.qr(torch.randn(n, n, dtype=f64, device=dev, generator=g))
    q2, _ = torch.linalg.qr(torch.randn(n, n, dtype=f64, device=dev, generator=g))
    sv = torch.logspace(0, -2, n, dtype=f64, device=dev)
    a_mixed = ((q1 * sv) @ q2.T).T.contiguous()
    del q1, q2
    a_mixed0 = a_mixed.clone()

    def mixed():
        AB.atlb_dsgesv_ex(n, 1, a_mixed, n, ipiv, b, n, x, n, 3, 0, it)
        if it[0] < 0:
            a_mixed.copy_(a_mixed0)

    search = [
        ("getrf_nb", [128, 192, 256], getrf, 3),
        ("lookahead", [0, 1], getrf, 3),
        ("lookahead_reserve_sms", [0, 8, 16], getrf, 3),
        ("potrf_nb", [128, 256, 384, 512], potrf, 3),
        ("dgemm_group", [4, 8, 16], dgemm_big, 3),
        ("dgemm_splitk", [0, 1], dgemm_small, 5),
        ("sgetrf_nb", [192, 224, 256], mixed, 7),
        ("mixed_tc_min_work_log2", [20, 22, 24, 26, 28, 31], mixed, 7),
    ]
    lines = [f"# atlas_b200 tuning, {time.strftime('%Y-%m-%d %H:%M:%S')}, "
             f"{torch.cuda.get_device_name(0)}, factorization order {n}"]
    for name, cands, fn, reps in search:
        times = {}
        for v in cands:
            AB.atlb_tune_set(name, v)
            times[v] = _timer(torch, stream, fn, reps)
        best = min(times, key=times.get)
        AB.atlb_tune_set(name, best)
        detail = ", ".join(f"{v}: {t:.3f} ms" for v, t in times.items())
        print(f"{name:>24} = {best:<6} ({detail})", flush=True)
        lines.append(f"# {name}: {detail}")
        lines.append(f"{name} {best}")
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
