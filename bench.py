"""Benchmark of the dense LU solve hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl atlas|reference]

Workload (one "step"): solve A x = b with N = 8192 (one right-hand side),
A = Q1 diag(s) Q2^T with Q1, Q2 from QR of Gaussian matrices and s geometric
from 1 to 1/kappa (kappa = 1e2), b uniform[-1, 1]; the solution must reach a
normwise backward error <= N * 2^-53.  Inputs are seeded synthetic data
generated on the device; they are larger than L2 (512 MiB), so no flush is
needed between steps.  Each step restores A from a pristine copy (the solver
overwrites it), like a caller that keeps its matrix.

Every rank runs an independent replica (the factorization of one matrix
does not shard); value = solves of all ranks / max-over-ranks time.

--impl reference times the reference's algorithm on the host cores: the
CPU restatement of ATLAS's recursive getrf + getrs (oracle/) on a bounded
sample (N = 2048), scaled to N = 8192 by the flop ratio.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dgesv N=8192 time @bwd err<=N*eps64: mixed vs FP64 GPU; DGEMM GFLOP/s vs peak"
N = 8192
KAPPA = 1e2


def lu_flops(n):
    # bin/lutst.c:267-269 (getrf) + 2 n^2 per right-hand side (getrs)
    return 2.0 / 3.0 * n ** 3 - 0.5 * n ** 2 + 2.0 * n ** 2


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import statistics
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, nm in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def make_system(torch, n, kappa, seed, dev):
    """A = Q1 diag(s) Q2^T (column-major storage), b ~ U[-1,1]."""
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    q1, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    q2, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    s = torch.logspace(0, -torch.log10(torch.tensor(kappa)).item(), n, dtype=torch.float64, device=dev)
    a = (q1 * s) @ q2.T                       # row-major logical A
    acol = a.T.contiguous()                   # storage of A in column-major order
    b = torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    del q1, q2
    return acol, b


def backward_error(torch, acol, x, b):
    """||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) with A column-major storage."""
    a = acol.T                                # logical A
    r = b - a @ x
    an = a.abs().sum(dim=1).max()
    return (r.abs().max() / (an * x.abs().max() + b.abs().max())).item()


def run_reference(args, rank, world):
    """CPU restatement of the reference's dgesv on host cores, bounded sample."""
    if rank != 0:
        return
    import numpy as np
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.orc().orc_set_threads(cores)
    ns = 2048
    a0 = O.lu_matrix(ns, 1)
    b0 = O.uniform((ns, 1), 2)
    times = []
    for i in range(args.warmup + args.steps):
        a = a0.copy(order="F")
        b = b0.copy(order="F")
        t0 = time.perf_counter()
        lu, ipiv, info = O.dgetrf(a)
        O.dgetrs(111, lu, ipiv, b)
        t1 = time.perf_counter()
        if i >= args.warmup:
            times.append(t1 - t0)
    t_sample = sum(times) / len(times)
    t_full = t_sample * lu_flops(N) / lu_flops(ns)
    val = 1.0 / t_full
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "solves/s (N=8192, 1 RHS)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_full * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": "dgesv N=8192, 1 RHS, FP64 (host CPU restatement of ATLAS getrfC+getrs)"},
        "cpu_baseline": {"value": val, "unit": "solves/s (N=8192, 1 RHS)", "cores": cores, "kind": "port",
                         "sample": f"dgesv N={ns} timed, scaled by flop ratio to N={N}"},
        "e2e": {"value": val, "unit": "solves/s (N=8192, 1 RHS)", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="atlas", choices=["atlas", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N, help="matrix order (default 8192; smaller for profiling)")
    ap.add_argument("--skip-e2e", action="store_true", help="omit the host-buffer leg (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    n = args.n

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import numpy as np
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import atlas_b200 as AB
    AB.lib()
    AB.atlb_init(local)
    # one non-default stream shared by torch (inputs, events) and the library
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    AB.atlb_set_stream(stream.cuda_stream)

    acol0, b0 = make_system(torch, n, KAPPA, 1234 + rank, dev)
    A = torch.empty_like(acol0)
    x = torch.empty_like(b0)
    ipiv = torch.empty(n, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    launches = {"n": 0}

    def step():
        A.copy_(acol0)
        x.copy_(b0)
        AB.atlb_dgetrf_dev(n, n, A, n, ipiv, info)
        AB.atlb_dgetrs_dev(111, n, 1, A, n, ipiv, x, n)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
        dist.barrier()
    berr = backward_error(torch, acol0, x, b0)
    assert int(info.item()) == 0
    value = world * 1000.0 / ms

    # mixed-precision solves of the same system (factor FP32 / TF32 / BF16, FP64 refinement)
    mixed = {}
    xm = torch.empty(n, dtype=torch.float64, device=dev)
    ipm = torch.empty(n, dtype=torch.int32, device=dev)
    it = np.zeros(1, dtype=np.int32)
    for name, prec in (("tf32", 1), ("bf16", 2), ("fp32", 0)):
        for _ in range(2):
            AB.atlb_dsgesv(n, 1, acol0, n, ipm, b0, n, xm, n, prec, it)
        ts = []
        for _ in range(max(2, args.steps // 2)):
            e0m, e1m = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0m.record(stream)
            r = AB.atlb_dsgesv(n, 1, acol0, n, ipm, b0, n, xm, n, prec, it)
            e1m.record(stream)
            torch.cuda.synchronize()
            ts.append(e0m.elapsed_time(e1m))
        mixed[name] = {"ms": sum(ts) / len(ts), "iter": int(it[0]), "info": int(r),
                       "backward_error": backward_error(torch, acol0, xm, b0)}

    # dominant kernel: the FP64 DMMA GEMM, timed alone at 8192^3
    M = 8192
    ga = torch.rand(M, M, dtype=torch.float64, device=dev) * 2 - 1
    gb = torch.rand(M, M, dtype=torch.float64, device=dev) * 2 - 1
    gc = torch.zeros(M, M, dtype=torch.float64, device=dev)
    for _ in range(2):
        AB.atlb_dgemm_dev(111, 111, M, M, M, 1.0, ga, M, gb, M, 0.0, gc, M)
    reps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        AB.atlb_dgemm_dev(111, 111, M, M, M, 1.0, ga, M, gb, M, 0.0, gc, M)
    e1.record(stream)
    torch.cuda.synchronize()
    dgemm_ms = e0.elapsed_time(e1) / reps
    dgemm_tf = 2.0 * M ** 3 / (dgemm_ms * 1e-3) / 1e12
    # measured FP64 denominator: cuBLAS DGEMM at the same size (library, denominator only)
    for _ in range(2):
        torch.matmul(ga, gb, out=gc)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        torch.matmul(ga, gb, out=gc)
    e1.record(stream)
    torch.cuda.synchronize()
    cublas_tf = 2.0 * M ** 3 / (e0.elapsed_time(e1) / reps * 1e-3) / 1e12
    del ga, gb, gc

    # end to end through the drop-in C ABI with pinned host buffers
    e2e_val = None
    if not args.skip_e2e:
        ha = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
        hb = torch.empty(n, dtype=torch.float64, pin_memory=True)
        ha_src = acol0.reshape(-1).cpu()
        hb_src = b0.cpu()
        hip = np.zeros(n, dtype=np.int32)
        e2e_t = []
        for i in range(2 + max(2, args.steps // 3)):
            ha.copy_(ha_src)
            hb.copy_(hb_src)
            t0 = time.perf_counter()
            r = AB.clapack_dgesv(AB.CblasColMajor, n, 1, ha, n, hip, hb, n)
            t1 = time.perf_counter()
            assert r == 0
            if i >= 2:
                e2e_t.append(t1 - t0)
        e2e_val = world / (sum(e2e_t) / len(e2e_t))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        O.orc().orc_set_threads(cores)
        ns = 1024
        a0 = O.lu_matrix(ns, 1)
        bb = O.uniform((ns, 1), 2)
        ts = []
        for _ in range(3):
            a = a0.copy(order="F")
            t0 = time.perf_counter()
            lu, ip, _ = O.dgetrf(a)
            O.dgetrs(111, lu, ip, bb.copy(order="F"))
            ts.append(time.perf_counter() - t0)
        tcpu = min(ts) * lu_flops(n) / lu_flops(ns)
        cpu = {"value": 1.0 / tcpu, "unit": "solves/s (N=8192, 1 RHS)", "cores": cores, "kind": "port",
               "sample": f"oracle getrf+getrs N={ns}, scaled by flop ratio to N={n}"}

    if rank == 0:
        gflops = lu_flops(n) / (ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s (N=8192, 1 RHS)", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, on device)",
            "config": {"workload": "dgesv N=8192 1 RHS, FP64 getrf+getrs (kappa=1e2 Q1 diag(s) Q2^T)",
                       "n": n, "nrhs": 1, "kappa": KAPPA, "parallelism": f"replicas x{world}",
                       "l2": "inputs 512 MiB > L2, no flush"},
            "fp64_dgesv_gflops": gflops, "mixed_dgesv": mixed, "backward_error": berr, "bwd_err_bound": n * 2.0 ** -53,
            "dgemm_8192": {"ms": dgemm_ms, "tflops": dgemm_tf, "cublas_fp64_tflops": cublas_tf},
            "roofline": {"bound": "tensor", "achieved": dgemm_tf, "peak": cublas_tf, "unit": "TFLOP/s",
                         "frac": dgemm_tf / cublas_tf, "traffic": None,
                         "peak_note": "FP64: no measured peak in MEASURED_PEAKS.json; denominator = cuBLAS DGEMM 8192^3 measured in this run"},
            "clocks": clk.summary(),
            "e2e": {"value": e2e_val, "unit": "solves/s (N=8192, 1 RHS)", "h2d_bytes_per_step": n * n * 8 + n * 8,
                    "d2h_bytes_per_step": n * n * 8 + n * 8 + n * 4},
            "cpu_baseline": cpu,
            "gpu_launches": None,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
