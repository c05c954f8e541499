"""Benchmark of the dense LU solve hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl atlas|reference]

Workload (one "step"): solve A x = b with N = 8192 (one right-hand side),
A = Q1 diag(s) Q2^T with Q1, Q2 from QR of Gaussian matrices and s geometric
from 1 to 1/kappa (kappa = 1e2), b uniform[-1, 1]; the solution must reach a
normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
<= N * 2^-53.  The headline `value` is the mixed-precision solver (FP32-class
factorization on the tensor cores + FP64 iterative refinement, library entry
atlb_dsgesv_ex); the plain FP64 GPU dgesv (getrf + getrs) on the same system
is reported beside it, with the speed-up.  Inputs are seeded synthetic data
generated on the device (larger than L2: 512 MiB, so no flush is needed).
The FP64 solver overwrites A, so each of its steps restores A from a copy.

Also reported: the FP64 DMMA DGEMM at 8192^3 (the roofline kernel, against
cuBLAS DGEMM measured in the same run) and the split-integer (Ozaki) DGEMM at
8192^3 with its error against a double-double oracle on a sampled block.

Every rank runs an independent replica (the factorization of one matrix
does not shard); value = solves of all ranks / max-over-ranks time.

--impl reference times the reference's algorithm on the host cores: the
CPU restatement of ATLAS's recursive getrf + getrs (oracle/, on all host
threads) solving the same N = 8192 system, whole solves, no extrapolation.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dgesv N=8192 time @bwd err<=N*eps64: mixed vs FP64 GPU; DGEMM GFLOP/s vs peak"
N_DEFAULT = 8192
KAPPA = 1e2
UNIT = "solves/s (N=8192, 1 RHS, bwd err <= N*2^-53)"
# headline mixed configuration: (name, factor precision, pivoting)
#   precision 0 FP32, 1 TF32, 2 BF16, 3 split TF32 (FP32-accurate); pivoting 0 partial, 1 RBT
HEADLINE = ("pp_tf32x3", 3, 0)
VARIANTS = [("rbt_tf32x3", 3, 1), ("rbt_tf32", 1, 1), ("rbt_fp32", 0, 1), ("pp_tf32x3", 3, 0),
            ("pp_tf32", 1, 0), ("pp_fp32", 0, 0), ("pp_bf16", 2, 0)]


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


def count_kernels(torch, fn):
    """Kernels one call of fn launches (CUPTI through torch.profiler; kernels
    inside replayed CUDA graphs are reported individually).  Returns
    (count, sorted distinct names) or (None, reason)."""
    try:
        from torch.profiler import profile, ProfilerActivity
        from torch.autograd import DeviceType
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events() if e.device_type == DeviceType.CUDA
                 and not e.name.startswith(("Memcpy", "Memset", "cudaMem"))]
        def short(n):  # "void ns::(anonymous namespace)::k<T, 32>(args)" -> "ns::k<T, 32>"
            n = n.replace("(anonymous namespace)::", "").replace("void ", "")
            return re.split(r"\((?!\d)", n)[0][:70]
        return len(names), sorted(set(short(n) for n in names))
    except Exception as exc:  # profiler unavailable on this box
        return None, repr(exc)[:120]


def backward_error(torch, acol, x, b):
    """||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) with A column-major storage."""
    a = acol.T                                # logical A
    r = b - a @ x
    an = a.abs().sum(dim=1).max()
    return (r.abs().max() / (an * x.abs().max() + b.abs().max())).item()


def replica_throughput(ms_local, world):
    """Whole-job solves/s of `world` independent replicas: every rank solved
    one system per step; the job's time per step is the slowest rank's
    (device time, MAX over ranks).  Returns (solves/s, ms per step)."""
    from atlas_b200 import parallel as PAR
    ms = PAR.max_over_ranks(ms_local)
    return world * 1000.0 / ms, ms


def host_system(n, kappa, seed):
    """The headline system as column-major host arrays (generated with torch on
    the GPU when there is one; the generation is not timed)."""
    import torch
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    acol, b = make_system(torch, n, kappa, seed, dev)
    a = np.asfortranarray(acol.cpu().numpy().reshape(n, n).T)   # logical A, column-major
    return a, np.asfortranarray(b.cpu().numpy().reshape(n, 1))


def cpu_dgesv(n, steps, warmup, budget_s):
    """FP64 dgesv (getrf + getrs) of the headline system on all host cores
    through the oracle -- the CPU restatement of the reference's recursive
    getrfC / laswp / getrs (oracle/atl_oracle.c) over its cache-blocked,
    threaded level-3 kernels (oracle/orc_fast.c).  Every timed solve is the
    full N x N problem; the number of timed solves is cut to fit budget_s.
    Returns (mean seconds per solve, solves timed, threads, backward error)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.orc().orc_set_threads(cores)
    a0, b0 = host_system(n, KAPPA, 1234)
    times = []
    x = None
    t_start = time.perf_counter()
    for i in range(warmup + steps):
        a = a0.copy(order="F")
        b = b0.copy(order="F")
        t0 = time.perf_counter()
        lu, ipiv, info = O.dgetrf(a)
        x = O.dgetrs(111, lu, ipiv, b)
        t1 = time.perf_counter()
        assert info == 0
        if i >= warmup:
            times.append(t1 - t0)
        elif t1 - t_start > budget_s / 2:      # a slow host: keep the warm-up short
            warmup = i + 1
        if times and (t1 - t_start) + (t1 - t0) > budget_s:
            break
    r = b0 - a0 @ x
    berr = float(np.max(np.abs(r)) / (np.max(np.sum(np.abs(a0), axis=1)) * np.max(np.abs(x))
                                      + np.max(np.abs(b0))))
    return sum(times) / len(times), len(times), cores, berr


def run_reference(args, rank, world):
    """The reference's dgesv on the host cores (the oracle's restatement of
    ATLAS's recursive getrfC + getrs), on the same system and config as the
    GPU arm: full N = 8192 solves, no extrapolation."""
    if rank != 0:
        return
    n = args.n
    t, done, cores, berr = cpu_dgesv(n, args.steps, args.warmup, budget_s=240.0)
    val = 1.0 / t
    sample = f"{done} timed full dgesv solves at N={n} (kappa={KAPPA:g}), {cores} host threads"
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": f"dgesv N={n} 1 RHS, FP64, kappa=1e2 Q1 diag(s) Q2^T "
                               "(host CPU restatement of ATLAS getrfC + getrs)",
                   "n": n, "nrhs": 1, "kappa": KAPPA},
        "backward_error": berr,
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed(torch, stream, fn, reps):
    """Mean ms of fn() over reps runs, CUDA events on the shared stream."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def measured_traffic(kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) that
    one ncu capture measured for `kernel`, from the data file kept beside the
    profile summaries (None when absent)."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("#") or "\t" not in line:
                continue
            name, val = line.rstrip("\n").split("\t")[:2]
            if name == kernel:
                return int(val)
    except OSError:
        pass
    return None


def peak_tf32_tflops():
    """Dense TF32 tensor peak: half the measured dense BF16 burst rate of this
    pool's B200s (MEASURED_PEAKS.json; the tensor cores run TF32 at half the
    BF16 rate), or half the fallback 1.59 PFLOP/s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)["bf16_tflops"] / 2.0, "half of measured bf16 burst (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 1590.0 / 2.0, "half of the fallback bf16 1.59 PFLOP/s"


def headline_roofline(torch, AB, dev, stream):
    """Roofline of the headline's tensor-core kernel: the split-TF32 GEMM of the
    FP32 factorization's first trailing update (M = 7936, N = 7680, K = 256;
    A and B each split into a TF32 high and a TF32 low plane, three products
    hi*hi + lo*hi + hi*lo on the tensor cores), timed with CUDA events on the
    library's stream over 10 calls
    (each call also runs the operand-split kernel).  Algorithmic work per call:
    2 * M * N * (3 K) TF32 flop.  Beside it, the latency of the FP32 leaf panel
    (one 8192 x 32 panel through atlb_sgetrf_dev) per column."""
    f32 = torch.float32
    M, N, K = 7936, 7680, 256
    g = torch.Generator(device=dev)
    g.manual_seed(77)
    a = torch.rand(K, M, dtype=f32, device=dev, generator=g) - 0.5   # column-major M x K
    b = torch.rand(N, K, dtype=f32, device=dev, generator=g) - 0.5   # column-major K x N
    c = torch.rand(N, M, dtype=f32, device=dev, generator=g) - 0.5
    call = lambda: AB.atlb_sgemm_tc_dev(3, 111, 111, M, N, K, -1.0, a, M, b, K, 1.0, c, M)
    for _ in range(3):
        call()
    ms = timed(torch, stream, call, 10)
    tflop = 2.0 * M * N * 3 * K / 1e12
    achieved = tflop / (ms / 1e3)
    peak, how = peak_tf32_tflops()
    # the leaf panel: one 8192 x 32 FP32 panel (partial pivoting)
    pn = 8192
    p = torch.rand(32, pn, dtype=f32, device=dev, generator=g) - 0.5
    p0 = p.clone()
    ip = torch.zeros(32, dtype=torch.int32, device=dev)
    inf = torch.zeros(1, dtype=torch.int32, device=dev)

    def panel():
        p.copy_(p0)
        AB.atlb_sgetrf_dev(pn, 32, p, pn, ip, inf, 0)
    for _ in range(3):
        panel()
    copy_ms = timed(torch, stream, lambda: p.copy_(p0), 10)
    panel_ms = timed(torch, stream, panel, 10) - copy_ms
    del a, b, c, p, p0
    name = "tc_gemm split-TF32 7936x7680x256"
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": measured_traffic(name), "kernel": name + " (2*M*N*3K TF32 flop per call)",
            "peak_note": how + "; of measured",
            "panel_us_per_column": panel_ms * 1e3 / 32,
            "panel_note": "FP32 leaf panel 8192 x 32 (fused partial-pivoting kernel), latency-bound"}


def extra_sharded(torch, AB, dev, stream, rank, world):
    """Paths that shard across GPUs (run when world > 1): DGEMM 8192^3 with C
    split into column slabs (A broadcast from rank 0 over NCCL inside the
    timed call, no other exchange), and the 10k batched SPD solves dealt out
    by work.  Times are device time, MAX over ranks."""
    from atlas_b200 import parallel as PAR
    f64 = torch.float64
    M = 8192
    g = torch.Generator(device=dev)
    g.manual_seed(99 + rank)
    a = torch.rand(M, M, dtype=f64, device=dev, generator=g) * 2 - 1
    s, w = PAR.column_slabs(M, world)[rank]
    b = torch.rand(max(w, 1), M, dtype=f64, device=dev, generator=g) * 2 - 1
    c = torch.zeros(max(w, 1), M, dtype=f64, device=dev)
    call = lambda: PAR.sharded_dgemm(a, b, c, M, M, M)
    for _ in range(2):
        call()
    ms = PAR.max_over_ranks(timed(torch, stream, call, 3))
    out = {"sharded_dgemm_8192": {"ms": ms, "tflops_all_ranks": 2.0 * M ** 3 / ms / 1e9, "ranks": world,
                                  "slab_of_rank0": list(PAR.column_slabs(M, world)[0]),
                                  "includes": "NCCL broadcast of A (512 MiB) + the rank's DGEMM slab"}}
    del a, b, c
    rng = np.random.default_rng(2024)
    sizes = rng.integers(8, 257, 10000).astype(np.int32)
    parts = PAR.split_by_work(sizes.astype(np.float64) ** 3 / 3 + 8.0 * sizes.astype(np.float64) ** 2, world)
    mine = parts[rank]
    As = [torch.eye(int(n), dtype=f64, device=dev) * (n + 1.0) for n in sizes[mine]]
    Bs = [torch.ones(4, int(n), dtype=f64, device=dev) for n in sizes[mine]]
    aptr = np.zeros(len(sizes), np.uint64)
    bptr = np.zeros(len(sizes), np.uint64)
    aptr[mine] = [t.data_ptr() for t in As]
    bptr[mine] = [t.data_ptr() for t in Bs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx, info = PAR.sharded_posv_batched(sizes, aptr, sizes, bptr, sizes, np.full(len(sizes), 4))
    t1 = time.perf_counter()
    out["sharded_posv_10k"] = {"ms_max_over_ranks": PAR.max_over_ranks((t1 - t0) * 1e3), "ranks": world,
                               "problems_rank0": int(len(parts[0])), "all_info_zero": bool(np.all(info == 0)),
                               "timing": "wall clock around the synchronous call"}
    return out


def extra_sgemm(torch, AB, dev, stream, M):
    """FP32 GEMM M^3: cblas_sgemm (the reference's entry point; FP32 FMA on the
    SIMT pipes, device pointers), cuBLAS FP32 with TF32 off in the same run,
    and the split-TF32 tensor-core product (atlb_sgemm_tc_dev precision 3).
    Errors: max |C - C_fp64| / max |C_fp64| on 256 rows of C."""
    f32 = torch.float32
    g = torch.Generator(device=dev)
    g.manual_seed(21)
    sa = torch.rand(M, M, dtype=f32, device=dev, generator=g) * 2 - 1   # column-major storage
    sb = torch.rand(M, M, dtype=f32, device=dev, generator=g) * 2 - 1
    sc = torch.zeros(M, M, dtype=f32, device=dev)
    rows = torch.arange(0, M, M // 256, device=dev)[:256]
    # column-major storage: logical A = sa^T, B = sb^T, C = sc^T; the sample is C[rows, :]
    ref = sa.T[rows].double() @ sb.T.double()
    flop = 2.0 * M ** 3

    def err():
        c_rows = sc.T[rows].double()
        return ((c_rows - ref).abs().max() / ref.abs().max()).item()

    out = {}
    simt = lambda: AB.cblas_sgemm(102, 111, 111, M, M, M, 1.0, sa, M, sb, M, 0.0, sc, M)
    for _ in range(2):
        simt()
    ms = timed(torch, stream, simt, 3)
    out["cblas_sgemm"] = {"ms": ms, "tflops": flop / ms / 1e9, "rel_err_vs_fp64": err(),
                          "path": "FP32 FMA on the SIMT pipes"}
    tc3 = lambda: AB.atlb_sgemm_tc_dev(3, 111, 111, M, M, M, 1.0, sa, M, sb, M, 0.0, sc, M)
    for _ in range(2):
        tc3()
    ms = timed(torch, stream, tc3, 3)
    out["split_tf32"] = {"ms": ms, "tflops": flop / ms / 1e9, "rel_err_vs_fp64": err(),
                         "path": "atlb_sgemm_tc_dev precision 3: hi*hi + lo*hi + hi*lo on tcgen05"}
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    # the storage of C = A B is sb @ sa (row-major), all contiguous
    for _ in range(2):
        torch.matmul(sb, sa, out=sc)
    ms = timed(torch, stream, lambda: torch.matmul(sb, sa, out=sc), 3)
    torch.backends.cuda.matmul.allow_tf32 = prev
    out["cublas_fp32"] = {"ms": ms, "tflops": flop / ms / 1e9, "rel_err_vs_fp64": err()}
    out["cblas_sgemm"]["frac_of_cublas_fp32"] = out["cblas_sgemm"]["tflops"] / out["cublas_fp32"]["tflops"]
    del sa, sb, sc
    return out


def extra_factorizations(torch, AB, dev, stream):
    """The FP64 factorization configurations: dgetrf+dgetrs N=8192 with 16
    right-hand sides on A = G/sqrt(N) + 4I, dpotrf+dpotrs N=8192 on
    A = G G^T/N + I, dgeqrf on a 16384 x 8192 Gaussian matrix."""
    f64 = torch.float64
    res = {}
    n, nrhs = 8192, 16
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    a0 = torch.randn(n, n, dtype=f64, device=dev, generator=g) / n ** 0.5
    a0 += 4.0 * torch.eye(n, dtype=f64, device=dev)
    b0 = torch.rand(nrhs, n, dtype=f64, device=dev, generator=g) * 2 - 1    # column-major n x nrhs
    A, B = torch.empty_like(a0), torch.empty_like(b0)
    ipiv = torch.zeros(n, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def lu():
        A.copy_(a0)
        B.copy_(b0)
        AB.atlb_dgetrf_dev(n, n, A, n, ipiv, info)
        AB.atlb_dgetrs_dev(111, n, nrhs, A, n, ipiv, B, n)
    lu()
    lu()
    ms = timed(torch, stream, lu, 3)
    flop = 2.0 / 3.0 * n ** 3 + 2.0 * n ** 2 * nrhs
    x = B.T                                   # logical n x nrhs
    r = b0.T - a0.T @ x
    resid = (r.abs().max() / (a0.abs().sum(0).max() * x.abs().max() * n * 2.0 ** -53)).item()
    res["dgetrf_dgetrs_8192_16rhs"] = {
        "ms": ms, "gflops": flop / ms / 1e6, "info": int(info.item()),
        "ipiv_identity": bool((ipiv == torch.arange(n, device=dev, dtype=torch.int32)).all().item()),
        "solve_residual_over_n_eps": resid}
    # Cholesky
    gm = torch.randn(n, n, dtype=f64, device=dev, generator=g)
    s0 = gm @ gm.T / n + torch.eye(n, dtype=f64, device=dev)
    del gm

    def ch():
        A.copy_(s0)
        B.copy_(b0)
        AB.atlb_dpotrf_dev(122, n, A, n, info)
        AB.atlb_dpotrs_dev(122, n, nrhs, A, n, B, n)
    ch()
    ch()
    ms = timed(torch, stream, ch, 3)
    flop = n ** 3 / 3.0 + 2.0 * n ** 2 * nrhs
    x = B.T
    r = b0.T - s0 @ x
    resid = (r.abs().max() / (s0.abs().sum(0).max() * x.abs().max() * n * 2.0 ** -53)).item()
    res["dpotrf_dpotrs_8192_16rhs"] = {"ms": ms, "gflops": flop / ms / 1e6, "info": int(info.item()),
                                       "solve_residual_over_n_eps": resid}
    del s0, A, B, a0, b0
    # QR
    m, nq = 16384, 8192
    q0 = torch.randn(nq, m, dtype=f64, device=dev, generator=g)             # column-major m x n
    Q = torch.empty_like(q0)
    tau = torch.empty(nq, dtype=f64, device=dev)

    def qr():
        Q.copy_(q0)
        AB.atlb_dgeqrf_dev(m, nq, Q, m, tau)
    qr()
    qr()   # the second call captures the factorization's graph; timed calls replay it
    ms = timed(torch, stream, qr, 2)
    flop = 2.0 * m * nq ** 2 - 2.0 / 3.0 * nq ** 3
    res["dgeqrf_16384x8192"] = {"ms": ms, "gflops": flop / ms / 1e6}
    del q0, Q
    torch.cuda.empty_cache()
    return res


def extra_kappa(torch, AB, dev, stream, n):
    """Mixed solver at kappa = 1e6: iterations (or FP64 fallback) per precision."""
    acol, b = make_system(torch, n, 1e6, 4321, dev)
    a0 = acol.clone()
    x = torch.empty_like(b)
    ipiv = torch.empty(n, dtype=torch.int32, device=dev)
    it = np.zeros(1, dtype=np.int32)
    res = {}
    for name, prec in (("fp32", 0), ("tf32x3", 3), ("bf16", 2)):
        def call():
            AB.atlb_dsgesv_ex(n, 1, acol, n, ipiv, b, n, x, n, prec, 0, it)
            if it[0] < 0:
                acol.copy_(a0)
        call()
        call()
        ms = timed(torch, stream, call, 2)
        res[name] = {"ms": ms, "iter": int(it[0]), "backward_error": backward_error(torch, a0, x, b)}
    del acol, a0
    return res


def extra_dsposv(torch, AB, dev, stream, n):
    """Mixed dsposv (split-TF32 Cholesky, FP64 refinement) on an SPD system
    A = Q diag(s) Q^T, s from 1 to 1/kappa (kappa = 1e2), b ~ U[-1, 1], device
    pointers; beside it the FP64 dpotrf + dpotrs on the same system."""
    g = torch.Generator(device=dev)
    g.manual_seed(777)
    q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))
    sv = torch.logspace(0, -2, n, dtype=torch.float64, device=dev)
    a = (q * sv) @ q.T
    a = 0.5 * (a + a.T)                       # symmetric: its storage is its column-major form
    del q
    b = torch.rand(n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    x = torch.empty_like(b)
    it = np.zeros(1, dtype=np.int32)

    def mixed():
        AB.atlb_dsposv(AB.CblasLower, n, 1, a, n, b, n, x, n, 3, it)
    mixed()
    mixed()
    ms = timed(torch, stream, mixed, 3)
    res = {"ms": ms, "iter": int(it[0]), "backward_error": backward_error(torch, a, x, b)}
    L = torch.empty_like(a)
    xf = torch.empty_like(b)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def fp64():
        L.copy_(a)
        xf.copy_(b)
        AB.atlb_dpotrf_dev(122, n, L, n, info)
        AB.atlb_dpotrs_dev(122, n, 1, L, n, xf, n)
    fp64()
    fp64()
    res["fp64_dpotrf_dpotrs_ms"] = timed(torch, stream, fp64, 3)
    res["fp64_backward_error"] = backward_error(torch, a, xf, b)
    res["speedup_mixed_vs_fp64"] = res["fp64_dpotrf_dpotrs_ms"] / ms
    res["system"] = "SPD Q diag(s) Q^T, kappa 1e2, 1 RHS, split-TF32 factors"
    del a, L
    return res


def extra_batched(torch, AB, dev, stream):
    """10,000 SPD systems (n in [8,256], 4 RHS), 10,000 LU solves, 50,000 uneven
    DGEMMs (M,N,K in [16,512]): one launch per batch, against a per-instance
    loop of the plain kernels on a sample of the same problems."""
    import ctypes
    f64 = torch.float64
    rng = np.random.default_rng(2024)
    res = {}

    def ptrs(ts):
        return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])

    count = 10000
    ns = rng.integers(8, 257, count).astype(np.int32)
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    # SPD A = B B^T + n I, generated per distinct size in batches
    As, Bs, A0s = [None] * count, [None] * count, [None] * count
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        gb = torch.randn(len(idx), n, n, dtype=f64, device=dev, generator=g)
        sp = gb @ gb.transpose(1, 2) + n * torch.eye(n, dtype=f64, device=dev)
        rh = torch.rand(len(idx), 4, n, dtype=f64, device=dev, generator=g) * 2 - 1
        for j, i in enumerate(idx):
            A0s[i] = sp[j]
            Bs[i] = rh[j]
    nr = np.full(count, 4, dtype=np.int32)
    info = np.zeros(count, dtype=np.int32)
    work = [a.clone() for a in A0s]
    rhs0 = [b.clone() for b in Bs]

    def posv():
        return AB.atlb_dposv_batched(count, ns, ptrs(work), ns, ptrs(Bs), ns, nr, info)
    # restore inputs outside the timed region, one timed launch at a time
    ts = []
    for rep in range(4):   # the third and later calls replay a captured graph
        for w, a in zip(work, A0s):
            w.copy_(a)
        for b, b0 in zip(Bs, rhs0):
            b.copy_(b0)
        ts.append(timed(torch, stream, lambda: posv(), 1))
    flop = float(np.sum(ns.astype(np.float64) ** 3 / 3 + 2.0 * ns.astype(np.float64) ** 2 * 4))
    batch_ms = min(ts[2:])
    sample = 300
    info_d = torch.zeros(1, dtype=torch.int32, device=dev)

    def loop():
        for i in range(sample):
            n = int(ns[i])
            AB.atlb_dpotrf_dev(122, n, work[i], n, info_d)
            AB.atlb_dpotrs_dev(122, n, 4, work[i], n, Bs[i], n)
    for w, a in zip(work[:sample], A0s[:sample]):
        w.copy_(a)
    loop()
    loop_ms = timed(torch, stream, loop, 1) * count / sample
    res["posv_10k"] = {"ms_one_launch": batch_ms, "gflops": flop / batch_ms / 1e6, "all_info_zero": bool((info == 0).all()),
                       "ms_per_instance_loop_scaled": loop_ms, "loop_sample": sample,
                       "speedup_vs_loop": loop_ms / batch_ms,
                       "timing": "CUDA events around the call (upload, launch, info back), graph replay"}
    del work, rhs0, A0s
    # LU solves: A = G/sqrt(n) + 4I, 1 RHS
    A0s, work = [None] * count, [None] * count
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        ga = torch.randn(len(idx), n, n, dtype=f64, device=dev, generator=g) / float(n) ** 0.5
        ga += 4.0 * torch.eye(n, dtype=f64, device=dev)
        for j, i in enumerate(idx):
            A0s[i] = ga[j]
    work = [a.clone() for a in A0s]
    rh = [torch.ones(1, int(n), dtype=f64, device=dev) for n in ns]
    piv = [torch.zeros(int(n), dtype=torch.int32, device=dev) for n in ns]
    one = np.ones(count, dtype=np.int32)
    ts = []
    for rep in range(4):
        for w, a in zip(work, A0s):
            w.copy_(a)
        ts.append(timed(torch, stream, lambda: AB.atlb_dgesv_batched(count, ns, ptrs(work), ns, ptrs(piv),
                                                                    ptrs(rh), ns, one, info), 1))
    batch_ms = min(ts[2:])
    flop = float(np.sum(2.0 / 3.0 * ns.astype(np.float64) ** 3 + 2.0 * ns.astype(np.float64) ** 2))
    # the factorization alone (the batched getrf configuration)
    tg = []
    for rep in range(4):
        for w, a in zip(work, A0s):
            w.copy_(a)
        tg.append(timed(torch, stream, lambda: AB.atlb_dgetrf_batched(count, ns, ptrs(work), ns, ptrs(piv), info), 1))
    getrf_ms = min(tg[2:])
    getrf_flop = float(np.sum(2.0 / 3.0 * ns.astype(np.float64) ** 3))
    res["getrf_10k"] = {"ms_one_launch": getrf_ms, "gflops": getrf_flop / getrf_ms / 1e6,
                        "all_info_zero": bool((info == 0).all()), "entry": "atlb_dgetrf_batched",
                        "timing": "CUDA events around the call (upload, launch, info back), graph replay"}
    for w, a in zip(work, A0s):
        w.copy_(a)

    def loop2():
        for i in range(sample):
            n = int(ns[i])
            AB.atlb_dgetrf_dev(n, n, work[i], n, piv[i], info_d)
            AB.atlb_dgetrs_dev(111, n, 1, work[i], n, piv[i], rh[i], n)
    loop2()
    loop_ms = timed(torch, stream, loop2, 1) * count / sample
    res["gesv_10k"] = {"ms_one_launch": batch_ms, "gflops": flop / batch_ms / 1e6, "all_info_zero": bool((info == 0).all()),
                       "ms_per_instance_loop_scaled": loop_ms, "loop_sample": sample,
                       "speedup_vs_loop": loop_ms / batch_ms,
                       "timing": "CUDA events around the call (upload, launch, info back), graph replay"}
    del work, A0s, rh, piv
    torch.cuda.empty_cache()
    # 50,000 uneven DGEMMs, every problem with its own A, B and C (about 84 GB
    # of operands, far beyond L2: the launch streams them from HBM)
    cnt = 50000
    M = rng.integers(16, 513, cnt).astype(np.int64)
    N = rng.integers(16, 513, cnt).astype(np.int64)
    K = rng.integers(16, 513, cnt).astype(np.int64)
    oa = np.concatenate([[0], np.cumsum(M * K)])
    ob = np.concatenate([[0], np.cumsum(K * N)])
    oc = np.concatenate([[0], np.cumsum(M * N)])
    abuf = torch.empty(int(oa[-1]), dtype=f64, device=dev)
    bbuf = torch.empty(int(ob[-1]), dtype=f64, device=dev)
    cbuf = torch.zeros(int(oc[-1]), dtype=f64, device=dev)
    for buf in (abuf, bbuf):   # generated in 1 Gi-element chunks
        for c0 in range(0, buf.numel(), 1 << 30):
            buf[c0:c0 + (1 << 30)].uniform_(-1.0, 1.0, generator=g)
    ap = (ctypes.c_void_p * cnt)(*[abuf.data_ptr() + 8 * int(o) for o in oa[:-1]])
    bp = (ctypes.c_void_p * cnt)(*[bbuf.data_ptr() + 8 * int(o) for o in ob[:-1]])
    cp = (ctypes.c_void_p * cnt)(*[cbuf.data_ptr() + 8 * int(o) for o in oc[:-1]])
    M32, N32, K32 = M.astype(np.int32), N.astype(np.int32), K.astype(np.int32)

    def grouped():
        return AB.atlb_dgemm_batched_dev(111, 111, cnt, M32, N32, K32, 1.0, ap, M32, bp, K32, 0.0, cp, M32)
    grouped()
    batch_ms = min(timed(torch, stream, grouped, 1) for _ in range(3))
    flop = float(np.sum(2.0 * M * N * K))
    algo_bytes = float(8 * np.sum(M * K + K * N + M * N))
    sample = 2000

    def loop3():
        for i in range(sample):
            AB.atlb_dgemm_dev(111, 111, int(M[i]), int(N[i]), int(K[i]), 1.0, ap[i], int(M[i]), bp[i], int(K[i]),
                              0.0, cp[i], int(M[i]))
    loop3()
    loop_ms = timed(torch, stream, loop3, 1) * cnt / sample
    res["dgemm_50k"] = {"ms_one_launch": batch_ms, "gflops": flop / batch_ms / 1e6,
                        "operand_gbytes": algo_bytes / 1e9, "operand_gb_per_s": algo_bytes / batch_ms / 1e6,
                        "ms_per_instance_loop_scaled": loop_ms, "loop_sample": sample,
                        "speedup_vs_loop": loop_ms / batch_ms,
                        "operands": "distinct A, B, C per problem (HBM-resident, beyond L2)",
                        "timing": "CUDA events"}
    del abuf, bbuf, cbuf
    torch.cuda.empty_cache()
    return res


def extra_adjoints(torch, AB, dev, stream):
    """Gaussian-likelihood loss adjoint at N=4096 (potrf/potrs adjoints) and
    the getrs adjoint, FP64; time of forward + adjoint."""
    f64 = torch.float64
    n = 4096
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    bm = torch.randn(n, n, dtype=f64, device=dev, generator=g)
    a = bm @ bm.T / n + torch.eye(n, dtype=f64, device=dev)
    del bm
    y = torch.rand(n, dtype=f64, device=dev, generator=g) * 2 - 1
    L, x = torch.empty_like(a), torch.empty_like(y)
    Lbar, Abar, Bbar = torch.zeros_like(a), torch.zeros_like(a), torch.empty_like(y)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def fwd_bwd():
        L.copy_(a)
        x.copy_(y)
        AB.atlb_dpotrf_dev(122, n, L, n, info)
        AB.atlb_dpotrs_dev(122, n, 1, L, n, x, n)
        Lbar.zero_()
        Lbar.view(-1)[:: n + 1] = 2.0 / L.view(-1)[:: n + 1]
        AB.atlb_dpotrf_adjoint_dev(n, L, n, Lbar, n, Abar, n)
        AB.atlb_dpotrs_adjoint_dev(n, 1, L, n, x, n, y, n, Bbar, n, Abar, n)
    fwd_bwd()
    fwd_bwd()   # graphs are captured on the second call and replayed from the third
    ms = timed(torch, stream, fwd_bwd, 3)
    ainv = torch.linalg.inv(a)
    av = ainv @ y
    closed = ainv - torch.outer(av, av)
    err = ((Abar - closed).abs().max() / closed.abs().max()).item()
    out = {"gaussian_loss_4096": {"ms_forward_plus_adjoint": ms, "rel_err_vs_closed_form": err}}
    del ainv, closed, L, Lbar
    # L(A) = c^T A^-1 b, A = G/sqrt(N) + 4I: getrf + getrs forward, the getrs adjoint
    ag = torch.randn(n, n, dtype=f64, device=dev, generator=g) / n ** 0.5 + 4.0 * torch.eye(n, dtype=f64, device=dev)
    acol = ag.T.contiguous()
    bv = torch.rand(n, dtype=f64, device=dev, generator=g) * 2 - 1
    cv = torch.rand(n, dtype=f64, device=dev, generator=g) * 2 - 1
    LU, xv, ipiv = torch.empty_like(acol), torch.empty_like(bv), torch.zeros(n, dtype=torch.int32, device=dev)
    Abar2 = torch.zeros_like(acol)

    def lu_fwd_bwd():
        LU.copy_(acol)
        xv.copy_(bv)
        AB.atlb_dgetrf_dev(n, n, LU, n, ipiv, info)
        AB.atlb_dgetrs_dev(111, n, 1, LU, n, ipiv, xv, n)
        Abar2.zero_()
        AB.atlb_dgetrs_adjoint_dev(n, 1, LU, n, ipiv, xv, n, cv, n, Bbar, n, Abar2, n)
    lu_fwd_bwd()
    lu_fwd_bwd()
    ms2 = timed(torch, stream, lu_fwd_bwd, 3)
    closed2 = -torch.outer(torch.linalg.solve(ag.T, cv), torch.linalg.solve(ag, bv))
    err2 = ((Abar2.T - closed2).abs().max() / closed2.abs().max()).item()
    out["getrs_adjoint_4096"] = {"ms_forward_plus_adjoint": ms2, "rel_err_vs_closed_form": err2,
                                 "loss": "c^T A^-1 b, A = G/sqrt(N) + 4I"}
    del ag, acol, LU, Abar2, closed2
    # the Gaussian loss of 512 systems at N = 128: batched forward (one launch) and
    # the two batched adjoints (one launch each)
    cnt, nb = 512, 128
    Bm = torch.randn(cnt, nb, nb, dtype=f64, device=dev, generator=g)
    A0 = Bm @ Bm.transpose(1, 2) / nb + torch.eye(nb, dtype=f64, device=dev)
    Ys = torch.rand(cnt, 1, nb, dtype=f64, device=dev, generator=g) * 2 - 1
    Lw, Xw = A0.clone(), Ys.clone()
    Lb = torch.zeros_like(A0)
    Ab3 = torch.zeros_like(A0)
    Bb3 = torch.zeros_like(Ys)
    pl = lambda t: np.array([t[i].data_ptr() for i in range(cnt)], dtype=np.uint64)
    nv = np.full(cnt, nb, np.int32)
    ones = np.ones(cnt, np.int32)
    inf3 = np.zeros(cnt, np.int32)
    pL, pX, pY, pLb, pAb, pBb = pl(Lw), pl(Xw), pl(Ys), pl(Lb), pl(Ab3), pl(Bb3)

    def batched_fwd_bwd():
        Lw.copy_(A0)
        Xw.copy_(Ys)
        AB.atlb_dposv_batched(cnt, nv, pL, nv, pX, nv, ones, inf3)
        Lb.zero_()
        Lb.diagonal(dim1=1, dim2=2).copy_(2.0 / Lw.diagonal(dim1=1, dim2=2))
        AB.atlb_dpotrf_adjoint_batched_dev(cnt, nv, pL, nv, pLb, nv, pAb, nv)
        AB.atlb_dpotrs_adjoint_batched_dev(cnt, nv, ones, pL, nv, pX, nv, pY, nv, pBb, nv, pAb, nv)
    batched_fwd_bwd()
    batched_fwd_bwd()
    ms3 = timed(torch, stream, batched_fwd_bwd, 3)
    ainv = torch.linalg.inv(A0)
    av = (ainv @ Ys.transpose(1, 2))[..., 0]
    closed3 = ainv - av[:, :, None] * av[:, None, :]
    err3 = ((Ab3.transpose(1, 2) - closed3).abs().amax() / closed3.abs().amax()).item()
    out["gaussian_loss_batched_512x128"] = {"ms_forward_plus_adjoint": ms3, "rel_err_vs_closed_form": err3,
                                            "launches": "batched posv + batched potrf adjoint + batched potrs adjoint"}
    return out


def run_probe(torch, AB, what, n, acol0, b0, x, ipiv, it, hprec, hpiv, dev, trace=False):
    """One call of a path between cudaProfilerStart/Stop, after two warm-up
    calls; with trace, the call's kernels from a CUPTI trace instead."""
    f64 = torch.float64
    if what in ("dgemm", "ozaki"):
        g = torch.Generator(device=dev)
        g.manual_seed(99)
        ga = torch.rand(n, n, dtype=f64, device=dev, generator=g) * 2 - 1
        gb = torch.rand(n, n, dtype=f64, device=dev, generator=g) * 2 - 1
        gc = torch.zeros(n, n, dtype=f64, device=dev)
        if what == "dgemm":
            call = lambda: AB.atlb_dgemm_dev(111, 111, n, n, n, 1.0, ga, n, gb, n, 0.0, gc, n)
        else:
            call = lambda: AB.atlb_dgemm_ozaki_dev(111, 111, n, n, n, 1.0, ga, n, gb, n, 0.0, gc, n, 8)
    elif what == "tcgemm":  # the headline roofline's split-TF32 GEMM (n is ignored)
        f32 = torch.float32
        M, N, K = 7936, 7680, 256
        g = torch.Generator(device=dev)
        g.manual_seed(77)
        a = torch.rand(K, M, dtype=f32, device=dev, generator=g) - 0.5
        b = torch.rand(N, K, dtype=f32, device=dev, generator=g) - 0.5
        c = torch.rand(N, M, dtype=f32, device=dev, generator=g) - 0.5
        call = lambda: AB.atlb_sgemm_tc_dev(3, 111, 111, M, N, K, -1.0, a, M, b, K, 1.0, c, M)
    elif what == "getrf":
        A = torch.empty_like(acol0)
        info = torch.zeros(1, dtype=torch.int32, device=dev)

        def call():
            A.copy_(acol0)
            AB.atlb_dgetrf_dev(n, n, A, n, ipiv, info)
    elif what == "potrf":   # dpotrf (lower) of an SPD matrix of order n
        g = torch.Generator(device=dev)
        g.manual_seed(5)
        gm = torch.randn(n, n, dtype=f64, device=dev, generator=g)
        S = gm @ gm.T / n + torch.eye(n, dtype=f64, device=dev)
        del gm
        A = torch.empty_like(S)
        info = torch.zeros(1, dtype=torch.int32, device=dev)

        def call():
            A.copy_(S)
            AB.atlb_dpotrf_dev(122, n, A, n, info)
    elif what == "geqrf":   # dgeqrf of a 2n x n Gaussian matrix
        g = torch.Generator(device=dev)
        g.manual_seed(5)
        G0 = torch.randn(n, 2 * n, dtype=f64, device=dev, generator=g)   # column-major 2n x n
        A = torch.empty_like(G0)
        tau = torch.zeros(n, dtype=f64, device=dev)

        def call():
            A.copy_(G0)
            AB.atlb_dgeqrf_dev(2 * n, n, A, 2 * n, tau)
    elif what == "mixed_posv":   # mixed dsposv on an SPD system (split-TF32 Cholesky), device pointers
        g = torch.Generator(device=dev)
        g.manual_seed(5)
        gm = torch.randn(n, n, dtype=f64, device=dev, generator=g)
        S = gm @ gm.T / n + torch.eye(n, dtype=f64, device=dev)
        del gm
        sx = torch.empty_like(b0)

        def call():
            AB.atlb_dsposv(AB.CblasLower, n, 1, S, n, b0, n, sx, n, hprec, it)
    elif what == "mixed_host":   # the e2e call: pinned host A, b, x (A copied while it is factored)
        ha = torch.empty((n, n), dtype=f64).pin_memory()
        ha.copy_(acol0.cpu())
        hb = torch.empty(n, dtype=f64).pin_memory()
        hb.copy_(b0.cpu())
        hx = torch.empty(n, dtype=f64).pin_memory()
        hpv = np.zeros(n, dtype=np.int32)

        def call():
            AB.atlb_dsgesv_ex(n, 1, ha, n, hpv, hb, n, hx, n, hprec, hpiv, it)
    else:
        a0 = acol0.clone()

        def call():
            AB.atlb_dsgesv_ex(n, 1, acol0, n, ipiv, b0, n, x, n, hprec, hpiv, it)
            if it[0] < 0:
                acol0.copy_(a0)
    call()
    call()
    torch.cuda.synchronize()
    if trace:
        print(json.dumps({"probe": what, "n": n, "trace": cupti_trace(torch, call)}), flush=True)
        return
    torch.cuda.profiler.start()
    call()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"probe": what, "n": n}), flush=True)


def cupti_trace(torch, call):
    """One call under torch.profiler (CUPTI activity records): the span from
    the first kernel's start to the last one's end, the time with at least one
    kernel running, and per stream the kernels' count and device time by name
    (the copy that resets the input included)."""
    import re
    from torch.profiler import profile, ProfilerActivity
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        call()
        torch.cuda.synchronize()
    ev = [e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
    ivs = sorted((e.time_range.start, e.time_range.end, e.name) for e in ev)
    if not ivs:
        return {}
    t0, t1 = ivs[0][0], max(e for _, e, _ in ivs)
    busy, cur_s, cur_e = 0.0, ivs[0][0], ivs[0][1]
    for s_, e_, _ in ivs[1:]:
        if s_ > cur_e:
            busy += cur_e - cur_s
            cur_s, cur_e = s_, e_
        else:
            cur_e = max(cur_e, e_)
    busy += cur_e - cur_s
    agg = {}
    for s_, e_, name in ivs:
        k = re.split(r"\((?!\d)", name.replace("(anonymous namespace)::", "").replace("atlb::", "")
                     .replace("void ", ""))[0][:70]
        a = agg.setdefault(k, [0, 0.0])
        a[0] += 1
        a[1] += e_ - s_
    top = sorted(agg.items(), key=lambda kv: -kv[1][1])
    return {"span_us": round(t1 - t0, 1), "busy_us": round(busy, 1),
            "kernel_us_total": round(sum(v[1] for _, v in top), 1),
            "kernels": [{"name": k, "launches": v[0], "us": round(v[1], 1), "avg_us": round(v[1] / v[0], 2)}
                        for k, v in top[:16]]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="atlas", choices=["atlas", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N_DEFAULT, help="matrix order (default 8192; smaller for profiling)")
    ap.add_argument("--skip-e2e", action="store_true", help="omit the host-buffer leg (profiling)")
    ap.add_argument("--skip-extras", action="store_true", help="only the headline and FP64 solves (profiling)")
    ap.add_argument("--probe", choices=["dgemm", "getrf", "potrf", "geqrf", "mixed", "mixed_host", "mixed_posv",
                                        "ozaki", "tcgemm"],
                    help="profiling aid: warm up, then run ONE call of the named path at order --n between "
                         "cudaProfilerStart/Stop (ncu --profile-from-start off) and exit")
    ap.add_argument("--trace", action="store_true",
                    help="with --probe: print the call's kernels (CUPTI trace: device time per kernel name, "
                         "span, busy time) instead of bracketing it for ncu")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    n = args.n

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
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
    # A solver that falls back to FP64 (LAPACK dsgesv: iter < 0) returns the
    # FP64 factors in A; the pristine copy restores it so every measurement
    # below solves the same system.
    apristine = acol0.clone()
    x = torch.empty_like(b0)
    ipiv = torch.empty(n, dtype=torch.int32, device=dev)
    it = np.zeros(1, dtype=np.int32)
    _, hprec, hpiv = HEADLINE
    if args.probe:
        return run_probe(torch, AB, args.probe, n, acol0, b0, x, ipiv, it, hprec, hpiv, dev, args.trace)

    fallbacks = [0]

    def mixed_step():
        r = AB.atlb_dsgesv_ex(n, 1, acol0, n, ipiv, b0, n, x, n, hprec, hpiv, it)
        assert r == 0
        if it[0] < 0:                 # the FP64 fallback ran: A holds its factors now
            fallbacks[0] += 1
            acol0.copy_(apristine)

    # ---- headline: mixed-precision solve, timed steps
    for _ in range(args.warmup):
        mixed_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fallbacks[0] = 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        torch.cuda.profiler.start()   # the timed region, for ncu --profile-from-start off
        ev0.record(stream)
        for _ in range(args.steps):
            mixed_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    value, ms = replica_throughput(ev0.elapsed_time(ev1) / args.steps, world)
    if world > 1:
        dist.barrier()
    per_step, kernel_names = count_kernels(torch, mixed_step)
    head_iter = int(it[0])
    head_berr = backward_error(torch, apristine, x, b0)

    # ---- plain FP64 GPU dgesv (getrf + getrs) on the same system
    A = torch.empty_like(acol0)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def fp64_step():
        A.copy_(apristine)
        x.copy_(b0)
        AB.atlb_dgetrf_dev(n, n, A, n, ipiv, info)
        AB.atlb_dgetrs_dev(111, n, 1, A, n, ipiv, x, n)

    for _ in range(2):
        fp64_step()
    fp64_ms = timed(torch, stream, fp64_step, max(2, args.steps // 2))
    assert int(info.item()) == 0
    fp64_berr = backward_error(torch, apristine, x, b0)
    del A

    out = {}
    if world > 1:
        out["multi_gpu"] = extra_sharded(torch, AB, dev, stream, rank, world)
    if not args.skip_extras:
        # ---- every mixed configuration (iterations, time, backward error)
        mixed = {}
        for name, prec, piv in VARIANTS:
            def call():
                AB.atlb_dsgesv_ex(n, 1, acol0, n, ipiv, b0, n, x, n, prec, piv, it)
                if it[0] < 0:
                    acol0.copy_(apristine)
            for _ in range(2):
                call()
            t_ms = timed(torch, stream, call, max(2, args.steps // 3))
            mixed[name] = {"ms": t_ms, "iter": int(it[0]),
                           "backward_error": backward_error(torch, apristine, x, b0)}
        out["mixed_variants"] = mixed

        # ---- the roofline kernel: FP64 DMMA DGEMM 8192^3 vs cuBLAS DGEMM (denominator)
        M = 8192
        flop = 2.0 * M ** 3
        ga = torch.rand(M, M, dtype=torch.float64, device=dev) * 2 - 1
        gb = torch.rand(M, M, dtype=torch.float64, device=dev) * 2 - 1
        gc = torch.zeros(M, M, dtype=torch.float64, device=dev)
        dg = lambda: AB.atlb_dgemm_dev(111, 111, M, M, M, 1.0, ga, M, gb, M, 0.0, gc, M)
        for _ in range(2):
            dg()
        dgemm_ms = timed(torch, stream, dg, 5)
        for _ in range(2):
            torch.matmul(ga, gb, out=gc)
        cublas_ms = timed(torch, stream, lambda: torch.matmul(ga, gb, out=gc), 5)
        dgemm_tf, cublas_tf = flop / dgemm_ms / 1e9, flop / cublas_ms / 1e9
        out["dgemm_8192"] = {"ms": dgemm_ms, "tflops": dgemm_tf, "cublas_fp64_tflops": cublas_tf,
                             "frac_of_cublas": dgemm_tf / cublas_tf,
                             "dram_bytes_per_launch": measured_traffic("dgemm_dmma_kernel 8192^3")}
        # the factorizations' trailing-update shape: C (8192 x 8192) -= A (8192 x K) B (K x 8192)
        short = {}
        for kk in (128, 192, 256):
            # column-major A (M x K, lda M) is a (K, M) tensor, B (K x N, ldb K) an (N, K) one
            sa, sb = ga[:kk, :].contiguous(), gb[:, :kk].contiguous()
            f_ours = lambda: AB.atlb_dgemm_dev(111, 111, M, M, kk, -1.0, sa, M, sb, kk, 1.0, gc, M)
            f_cub = lambda: torch.addmm(gc, sb, sa, alpha=-1.0, out=gc)
            for f in (f_ours, f_cub):
                f()
            t_ours, t_cub = timed(torch, stream, f_ours, 5), timed(torch, stream, f_cub, 5)
            fl = 2.0 * M * M * kk
            short[f"k{kk}"] = {"tflops": fl / t_ours / 1e9, "cublas_fp64_tflops": fl / t_cub / 1e9}
        out["dgemm_8192_short_k"] = short
        del ga, gb
        out["sgemm_8192"] = extra_sgemm(torch, AB, dev, stream, M)
        out["roofline"] = headline_roofline(torch, AB, dev, stream)

        # ---- split-integer (Ozaki) DGEMM 8192^3 on the INT8 tensor cores
        # operands x = u * 2^e, u ~ U[-1,1], e ~ U{-10..10}; storage tensors hold
        # the column-major matrices, i.e. logical A = oa^T, B = ob^T, C = gc^T
        g = torch.Generator(device=dev)
        g.manual_seed(99)
        oa = (torch.rand(M, M, dtype=torch.float64, device=dev, generator=g) * 2 - 1) * \
            torch.exp2(torch.randint(-10, 11, (M, M), device=dev, generator=g).double())
        ob = (torch.rand(M, M, dtype=torch.float64, device=dev, generator=g) * 2 - 1) * \
            torch.exp2(torch.randint(-10, 11, (M, M), device=dev, generator=g).double())
        from oracle import oracle as O
        O.orc().orc_set_threads(os.cpu_count() or 1)
        idx = torch.arange(0, M, M // 48, device=dev)[:48]
        a_rows = np.asfortranarray(oa[:, idx].T.cpu().numpy())     # A[idx, :]
        b_cols = np.asfortranarray(ob[idx, :].T.cpu().numpy())     # B[:, idx]
        hi, lo = O.ddgemm(a_rows, b_cols)                          # double-double C[idx, idx]

        def block(c):
            return np.asfortranarray(c[idx][:, idx].T.cpu().numpy())

        AB.atlb_dgemm_dev(111, 111, M, M, M, 1.0, oa, M, ob, M, 0.0, gc, M)
        oz = {"plain_fp64_err": O.normwise_err_dd(block(gc), hi, lo),
              "sample": "48x48 block of C vs double-double oracle"}
        for s in (6, 7, 8):
            f = lambda: AB.atlb_dgemm_ozaki_dev(111, 111, M, M, M, 1.0, oa, M, ob, M, 0.0, gc, M, s)
            f()
            t_ms = timed(torch, stream, f, 3)
            oz[f"slices{s}"] = {"ms": t_ms, "effective_tflops": flop / t_ms / 1e9,
                                 "err_vs_dd": O.normwise_err_dd(block(gc), hi, lo),
                                 "speedup_vs_dmma_dgemm": dgemm_ms / t_ms}
        out["ozaki_8192"] = oz
        del gc, oa, ob
        torch.cuda.empty_cache()
        out["fp64_factorizations"] = extra_factorizations(torch, AB, dev, stream)
        out["mixed_kappa_1e6"] = extra_kappa(torch, AB, dev, stream, n)
        out["mixed_dsposv_8192"] = extra_dsposv(torch, AB, dev, stream, n)
        out["batched"] = extra_batched(torch, AB, dev, stream)
        out["adjoints"] = extra_adjoints(torch, AB, dev, stream)

    # ---- end to end through the C ABI with pinned host buffers (H2D of A and b,
    # D2H of x inside the timed region)
    e2e = None
    if not args.skip_e2e:
        ha = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
        hb = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hx = torch.empty(n, dtype=torch.float64, pin_memory=True)
        ha.copy_(apristine.reshape(-1).cpu())
        hb.copy_(b0.cpu())
        hip = np.zeros(n, dtype=np.int32)
        e2e_t = []
        for i in range(2 + max(2, args.steps // 3)):
            t0 = time.perf_counter()
            r = AB.atlb_dsgesv_ex(n, 1, ha, n, hip, hb, n, hx, n, hprec, hpiv, it)
            t1 = time.perf_counter()
            assert r == 0
            if it[0] < 0:
                ha.copy_(apristine.reshape(-1).cpu())
            if i >= 2:
                e2e_t.append(t1 - t0)
        e2e = {"value": world / (sum(e2e_t) / len(e2e_t)), "unit": UNIT,
               "h2d_bytes_per_step": n * n * 8 + n * 8, "d2h_bytes_per_step": n * 8,
               "path": "atlb_dsgesv_ex with pinned host A, b, x"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t, done, cores, berr = cpu_dgesv(n, 3, 1, budget_s=30.0)
        cpu = {"value": 1.0 / t, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{done} timed full dgesv solves at N={n} (oracle getrfC + getrs, "
                         f"{cores} host threads), backward error {berr:.2e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, on device)",
            "config": {"workload": f"mixed dgesv N={n} 1 RHS ({HEADLINE[0]}) vs FP64 dgesv, kappa=1e2 Q1 diag(s) Q2^T",
                       "n": n, "nrhs": 1, "kappa": KAPPA, "parallelism": f"replicas x{world}",
                       "l2": "inputs 512 MiB > L2, no flush"},
            "headline": {"solver": HEADLINE[0], "ms": ms, "iter": head_iter, "backward_error": head_berr,
                         "fp64_fallbacks_in_timed_steps": fallbacks[0],
                         "bwd_err_bound": n * 2.0 ** -53},
            "fp64_dgesv": {"ms": fp64_ms, "gflops": lu_flops(n) / fp64_ms / 1e6, "backward_error": fp64_berr},
            "speedup_mixed_vs_fp64": fp64_ms / ms,
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": None if per_step is None else per_step * args.steps,
            "gpu_launches_note": ("kernels of one headline step counted with CUPTI (torch.profiler) "
                                  "after the timed region, times steps"),
            "kernels_per_step": per_step,
            "kernel_names": kernel_names,
        }
        line.update(out)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
