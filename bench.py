#!/usr/bin/env python
"""Benchmark of the harmonic-conversion hot path on B200.

Headline workload (one "step"): sph2fourier('N') followed by fourier2sph('N') on
16 fields of degree 4095 sharing one plan (n = 4096 rows, M = 8191 columns each,
column-major), seeded U(-1,1) in the reference's triangular sph layout, through
ft_b200_execute_shared_dev with the split-BF16 tensor-core path (MIXED_BF16:
three 9-bit slices per operand in the blocked sweeps).  Metric: coefficients per second, fields * n^2 / (t_fwd + t_bwd),
reported beside the plain FP64 GPU path on the same fields (their ratio) and the
relative 2-norm / max errors of the mixed result against the FP64 transform.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 4096] [--fields 16]

Under torchrun (N > 1) every rank runs an independent replica on its own
fields (the path has no exchange step); the step time is the max over ranks.

Arms:
  ours       the CUDA library: device-resident timing (value), roofline of the
             dominant kernel from CUDA events recorded around each launch on its
             stream, end-to-end timing with the fields copied from and to pinned
             host memory inside the timed region (e2e), and the reference's CPU
             build timed on a sample of the same workload; the secondary
             workloads (plain FP64 single field, the full spherical-harmonic
             transform with the grid stage, the spin-weighted transform, uneven
             batch, every precision of the shared-plan call, tri / disk) follow
             under "workloads".
  reference  the reference FastTransforms library compiled from its own sources
             (oracle/_ref/libft_ref.so, OpenMP + its AVX kernels + OpenBLAS), run
             on the host cores, one field of the workload per step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sph2fourier fwd+bwd coeffs/s: batched mixed-prec vs plain FP64 GPU, ε₂≤1e-6"
UNIT = "coeffs/s"
SEED = 20261203


def rotations_sph(n: int) -> int:
    """Givens rotations of one sph hi2lo (or lo2hi) over all orders (src/drivers.c:94-101)."""
    tot = 0
    for m in range(2, n):
        c = m // 2                       # sweeps j = m-2, m-4, ..., m % 2
        sum_j = c * (m % 2 + m - 2) // 2
        tot += 2 * (c * (n - 2) - sum_j)  # sweep j rotates rows k = 0 .. n-3-j, both columns
    return tot


def trmm_flops(n: int, M: int) -> int:
    """Upper-triangular multiply of all M columns: n(n+1)/2 multiply-adds per column."""
    return n * (n + 1) * M


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except Exception:
        return {}


def fp64_peak_tflops(torch) -> float:
    """cuBLAS DGEMM 8192^3 burst (best of 5), the FP64 counterpart of the bf16 GEMM peak."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", gpu_id], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_cpu():
    """(threads, description): the reference runs one OpenMP / BLAS thread per physical core
    available to this process; the description names the CPU model and the counts."""
    avail = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    logical = os.cpu_count() or avail
    try:
        import psutil
        physical = psutil.cpu_count(logical=False) or logical
    except Exception:
        physical = logical
    per_core = max(1, logical // max(physical, 1))
    threads = max(1, avail // per_core)
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return threads, (f"{model}; {avail} logical CPUs available ({logical} on the host, {physical} physical cores), "
                     f"{threads} threads = one per available physical core")


def ft_time(block, ntimes: int) -> float:
    """The reference's FT_TIME (src/ftutilities.h:15-21): two untimed runs of the block, then
    the mean over ntimes timed runs."""
    block()
    block()
    t0 = time.perf_counter()
    for _ in range(ntimes):
        block()
    return (time.perf_counter() - t0) / ntimes


def quad_cols(M: int) -> list:
    """Columns of every stride-4 class spread over all orders, where the GPU's forward transforms
    are compared with the quad-precision oracle (the same set as the parity tests)."""
    return sorted({0, 1, 2, 3, 4, 5, 6, M // 4 - 1, M // 4, M // 4 + 1, M // 4 + 2, M // 2 - 1, M // 2, M // 2 + 1,
                   M // 2 + 2, 3 * M // 4, 3 * M // 4 + 1, M - 4, M - 3, M - 2, M - 1})


def cpu_sample(n: int, ref_out: str | None = None) -> dict:
    """Reference CPU build on this host's cores with the reference's timing protocol:
    FT_TIME (two warm-ups, then NTIMES = 1 + (2048 / n)^2 timed runs in C integer arithmetic,
    test/test_drivers.c:257) of sph2fourier 'N' and of fourier2sph 'N', each repeated five times,
    the medians summed.  With ref_out, the reference's forward 'N' of the field (before any
    timing) is saved there for the GPU's parity check, and beside it (ref_out + ".quad.npy") the
    __float128 oracle's forward of the same field on quad_cols(M), with the reference plan's own
    connection matrices (oracle/ft_quad.c; a checker, run here on the host only)."""
    import numpy as np
    threads, cpu_desc = host_cpu()
    from oracle.bind import Reference, Oracle, fill
    A = fill("sph", n, SEED)
    if Reference.available():
        R = Reference()
        kind = "reference"
        R.set_num_threads(threads)
        P = R.plan("sph", n)
        run = lambda fwd, B: R.execute("sph", P, fwd, "N", B)
    else:
        R = Oracle()
        kind = "port"
        P = R.plan("sph", n)
        run = lambda fwd, B: R.execute(P, fwd, "N", B)
    if ref_out:
        F = A.copy(order="F")
        run(True, F)
        np.save(ref_out, F)
        del F
        if kind == "reference":
            from oracle.bind import Quad
            Ps, _ = R.connection(P, n)
            hi, _ = Quad().columns("sph", A, quad_cols(A.shape[1]), (), True, (np.triu(Ps[0]), np.triu(Ps[1])))
            np.save(ref_out + ".quad.npy", hi)
            del Ps
    ntimes = 1 + (2048 // n) ** 2
    B = A.copy(order="F")
    tf = statistics.median(ft_time(lambda: run(True, B), ntimes) for _ in range(5))
    tb = statistics.median(ft_time(lambda: run(False, B), ntimes) for _ in range(5))
    R.destroy(P)
    t = tf + tb
    res = {"value": n * n / t, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"sph n={n} (degree {n - 1}), 1 field: FT_TIME (2 warm-ups + NTIMES={ntimes}) of sph2fourier 'N' "
                     f"and of fourier2sph 'N', median of 5 each, summed; OMP threads = OpenBLAS threads = {threads}; "
                     f"reference built from its own sources: per-ISA kernel files at the reference's Make.inc flags "
                     f"with cpuid dispatch (AVX-512F kernels where the CPU has them), generic sources at "
                     f"-O3 -march=x86-64-v3 (not -march=native, so the one build runs on every host)",
           "cpu": cpu_desc, "sec_per_step": t, "sec_fwd": tf, "sec_bwd": tb}
    if kind == "reference":
        # the spin-weighted transform (s = 2) beside the GPU's spin workload: one timed
        # fwd+bwd 'N' after one warm-up
        from oracle.bind import fill_spin
        s = 2
        Z = fill_spin(n, 2 * n - 1, s, SEED)
        SP = R.spin_plan(n, s)
        R.spin_execute(SP, True, "N", Z)
        R.spin_execute(SP, False, "N", Z)
        t0 = time.perf_counter()
        R.spin_execute(SP, True, "N", Z)
        R.spin_execute(SP, False, "N", Z)
        ts = time.perf_counter() - t0
        R.spin_destroy(SP)
        res["spin_s2"] = {"value": n * n / ts, "sec_per_step": ts, "cores": threads,
                          "sample": f"spinsph2fourier + fourier2spinsph 'N', s = {s}, n={n}, 1 complex field, "
                                    f"1 timed after 1 warm-up"}
        # the other families beside the GPU's family workloads: one timed fwd+bwd 'N' after one warm-up
        from oracle.bind import fill as fill2
        from fasttransforms_b200.utilities import tetrand, rectdiskrand

        def once(run):
            run()
            t0 = time.perf_counter()
            run()
            return time.perf_counter() - t0
        fam = {}
        try:
            P = R.plan("rect", 4096, beta=0.0)
            Z = rectdiskrand(4096, SEED)
            t = once(lambda: (R.execute("rect", P, True, "N", Z), R.execute("rect", P, False, "N", Z)))
            R.destroy(P)
            fam["rectdisk_n4096"] = {"value": 4096 * 4097 // 2 / t, "sec_per_step": t}
            rho = float(np.sqrt(1 / 3))
            P = R.ann_plan(2048, 0.0, 0.0, rho)
            Z = fill2("disk", 2048, SEED)
            t = once(lambda: (R.ann_execute(P, True, "N", Z), R.ann_execute(P, False, "N", Z)))
            R.destroy(P)
            fam["ann_n2048"] = {"value": (2 * 2048 * 2048 - 2048) / t, "sec_per_step": t}
            P = R.tet_plan(256, 0.0, 0.0, 0.0, 0.0)
            Z = tetrand(256, SEED)
            t = once(lambda: (R.tet_execute(P, True, "N", Z), R.tet_execute(P, False, "N", Z)))
            R.destroy(P)
            fam["tet_n256"] = {"value": 256 * 257 * 258 // 6 / t, "sec_per_step": t}
        except Exception as exc:
            fam["error"] = repr(exc)[:200]
        res["families"] = fam
    return res


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads, cpu_desc = host_cpu()
    os.environ["OMP_NUM_THREADS"] = os.environ["OPENBLAS_NUM_THREADS"] = str(threads)   # read when the library loads
    from oracle.bind import Reference, fill
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libft_ref.so was not built"}))
        return
    n = args.n
    M = 2 * n - 1
    R = Reference()
    R.set_num_threads(threads)
    P = R.plan("sph", n)
    A = fill("sph", n, SEED)
    for _ in range(args.warmup):
        R.execute("sph", P, True, "N", A)
        R.execute("sph", P, False, "N", A)
    ts = []
    budget = 240.0
    t_all = time.perf_counter()
    for k in range(args.steps):
        t0 = time.perf_counter()
        R.execute("sph", P, True, "N", A)
        R.execute("sph", P, False, "N", A)
        ts.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget:
            break
    R.destroy(P)
    tot = sum(ts)
    value = n * n * len(ts) / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": len(ts), "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(ts),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded U(-1,1) in the sph triangular layout",
            "config": {"workload": f"sph2fourier+fourier2sph FP64, degree {n - 1} (n={n}, M={M}), host CPU; "
                                   f"each step is one of the {args.fields} fields of the shared-plan workload",
                       "n": n, "fields_per_step": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{len(ts)} steps of one field each (the reference has no batch call; a field "
                                       f"is the workload's unit), OMP threads = BLAS threads = {threads}; reference "
                                       f"built from its own sources (per-ISA kernels with cpuid dispatch, generic "
                                       f"sources at -O3 -march=x86-64-v3)",
                             "cpu": cpu_desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def profiled_traffic(workload, kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel` on
    `workload`, from the table of ncu figures kept in profiles/traffic.txt (None if absent)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == workload and f[1] == kernel:
            try:
                return float(f[2])
            except ValueError:
                return None
    return None


def max_over_ranks(x: float, dist, device: str) -> float:
    """The largest of every rank's x (each rank times its own replica; the job's time is the
    slowest rank's).  dist None: single process."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(coeffs_per_rank: int, world: int, steps: int, ms: float) -> float:
    """Whole-job coefficients per second: every rank transforms its own fields each step."""
    return world * coeffs_per_rank * steps / (ms * 1e-3)


def block_split_rotations(n: int, blk: int = 32):
    """Rotations of one sph hi2lo over all orders, split into those of whole blocks of
    `blk` sweeps (the tensor-core products) and the heads above them (direct kernel)."""
    heads = blocks = 0
    for m in range(2, n):
        p = m % 2
        h = ((m - p) // 2) % blk                 # head sweeps j = m-2, ..., m - 2h
        for j in range(m - 2, p - 1, -2):
            r = 2 * (n - 2 - j)
            if j >= m - 2 * h:
                heads += r
            else:
                blocks += r
    return blocks, heads


def block_tiles(n: int, nf: int, blk: int = 32, tl: int = 32) -> int:
    """Tile products (128 columns x both chains each) of the blocked stage for nf fields."""
    mlast = n - 1
    nbeta = (n - 1) // (2 * blk)

    def kmax(p, beta):
        j0 = p + 2 * blk * beta + 2 * blk - 2
        x = n - 3 - j0
        t0 = x // 2 if x >= 0 else -((1 - x) // 2)
        return t0 // tl if t0 >= 0 else -1
    tiles = 0
    for p in range(2):
        band = 1
        while p + 2 * blk * band <= mlast:
            if band <= nbeta:
                tiles += sum(kmax(p, b) + 2 for b in range(band))
            band += 1
    return tiles * ((nf + 1) // 2)


def run_ours(args, rank, world, local_rank, dist):
    import numpy as np
    import torch
    import fasttransforms_b200 as ft

    torch.cuda.set_device(local_rank)
    dev = torch.cuda.current_device()
    props = torch.cuda.get_device_properties(dev)
    n, nf = args.n, args.fields
    M = 2 * n - 1
    prec = ft.MIXED_BF16
    P = ft.plan_sph2fourier(n)
    host = [ft.sphrand(n, SEED + rank * nf + f) for f in range(nf)]
    d = [torch.from_numpy(A.ravel(order="F").copy()).cuda() for A in host]
    ptrs = [t.data_ptr() for t in d]
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def step(pr=prec):
        ft.execute_shared_dev(P, True, "N", ptrs, pr, sptr)
        ft.execute_shared_dev(P, False, "N", ptrs, pr, sptr)

    def reset():
        for t, A in zip(d, host):
            t.copy_(torch.from_numpy(A.ravel(order="F")))

    # accuracy against the FP64 transform (the direct FP64 path, parity-pinned to the
    # oracle at 1e-14): forward and round trip, all fields (builds every table first)
    ft.execute_shared_dev(P, True, "N", ptrs, ft.FP64, sptr)
    ref_fwd = [t.clone() for t in d]
    fp64_f0 = ref_fwd[0].cpu().numpy() if rank == 0 else None    # field 0, for the parity check against the reference
    reset()
    ft.execute_shared_dev(P, True, "N", ptrs, prec, sptr)
    mixed_f0 = d[0].cpu().numpy() if rank == 0 else None
    fw = torch.cat(d)
    rf = torch.cat(ref_fwd)
    eps2 = float(torch.linalg.norm(fw - rf) / torch.linalg.norm(rf))
    epsinf = float((fw - rf).abs().max() / rf.abs().max())
    del fw, rf, ref_fwd
    ft.execute_shared_dev(P, False, "N", ptrs, prec, sptr)
    back = torch.cat(d)
    src = torch.cat([torch.from_numpy(A.ravel(order="F")) for A in host]).cuda()
    rt2 = float(torch.linalg.norm(back - src) / torch.linalg.norm(src))
    rtinf = float((back - src).abs().max() / src.abs().max())
    del back, src
    status = ft.device_status(P)
    reset()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    uuid = getattr(props, "uuid", None)
    gpu_id = ("GPU-" + str(uuid)) if uuid is not None else str(local_rank)
    sampler = ClockSampler(gpu_id)
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ft.kernel_launches()
    ft.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    launches = ft.kernel_launches() - launches0
    fam = {name: ft.profile_read(i) for i, name in enumerate(("heads", "trmm", "transposes", "blocks"))}
    ft.profile(False)
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, dist, "cuda")
    coeffs = nf * n * n
    value = replica_value(coeffs, world, args.steps, ms)

    # the same fields through the plain FP64 path
    psteps = max(2, args.steps // 3)
    for _ in range(2):
        step(ft.FP64)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0.record(stream)
    for _ in range(psteps):
        step(ft.FP64)
    e1.record(stream)
    torch.cuda.synchronize()
    pms = e0.elapsed_time(e1)
    pms = max_over_ranks(pms, dist, "cuda")
    plain_value = replica_value(coeffs, world, psteps, pms)

    # end to end through the C-ABI call ft_b200_execute_shared_host: every step the fields start
    # in page-locked host memory, go to the device in groups (copies overlapped with the
    # transforms of the previous group), run forward and backward, and come back
    hb = [torch.from_numpy(A.ravel(order="F").copy()).pin_memory() for A in host]
    hptr = [h.data_ptr() for h in hb]
    ops = [(True, "N"), (False, "N")]
    e2e_steps = max(1, min(args.steps, 4))
    del d                                     # the pipeline's own device buffers replace them
    torch.cuda.empty_cache()
    ft.execute_shared_host(P, ops, hptr, prec)   # first call: allocates the pipeline's buffers
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ft.execute_shared_host(P, ops, hptr, prec)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    e2e_value = world * coeffs * e2e_steps / e2e_s
    bytes_mat = n * M * 8
    del hb

    if rank != 0:
        P.close()
        return
    # roofline of the dominant kernel: the split-BF16 tile products of the blocked sweeps
    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(torch)
    bf16 = peaks.get("bf16_tflops") or 1590.0
    bf16_sus = peaks.get("bf16_tflops_sustained") or 1400.0
    peak_src = "MEASURED_PEAKS.json" if peaks.get("bf16_tflops_sustained") else "fallback (no MEASURED_PEAKS.json)"
    rb, rh = block_split_rotations(n)
    blk_ms, blk_n = fam["blocks"]
    per_launch = blk_ms / max(blk_n, 1)
    alg_flops = 6 * rb * nf                                     # algorithmic: the rotations the blocks apply
    tiles = block_tiles(n, nf)
    products = 8                                                # three slices, levels <= 3
    issued = tiles * 2 * products * 2 * 128 * 64 * 64           # MMA flops the kernel issues
    achieved = alg_flops / (per_launch * 1e-3) / 1e12
    # peak: the split-BF16 emulation of FP64-class work at three BF16 products per product, against
    # the sustained BF16 GEMM rate (the kernel runs inside a seconds-long timed region)
    alg_peak = bf16_sus / 3.0
    # secondary: the algorithmic rate at which this design saturates the tensor pipe (its eight
    # slice products and the 4/3 of a 64 x 64 tile product over its 32 x 32 rotations)
    pipe_rate = bf16 / (products * 4.0 / 3.0)
    traffic = profiled_traffic(f"shared{nf}_n{n}", "blocked_mixed_kernel")
    roofline = {
        "bound": "tensor", "kernel": "blocked_mixed_kernel (tcgen05 split-BF16 tile products, 3 slices)",
        "achieved": achieved, "peak": alg_peak, "unit": "TFLOP/s", "frac": achieved / alg_peak, "traffic": traffic,
        "peak_source": f"{peak_src} bf16_tflops_sustained {bf16_sus} / 3 (three BF16 products per emulated product); "
                       f"achieved = algorithmic flops (6 per rotation the blocks apply) / mean launch time",
        "frac_of_design_pipe_rate": achieved / pipe_rate,
        "design_pipe_rate_tflops": pipe_rate,
        "design_pipe_rate_source": f"bf16_tflops {bf16} (burst) / (8 slice products x 4/3 tile overhead)",
        "algorithmic_flops_per_launch": alg_flops, "ms_per_launch": per_launch,
        "tensor_flops_issued_per_launch": issued,
        "tensor_pipe_frac": issued / (per_launch * 1e-3) / 1e12 / bf16,
        "fp64_equivalent_frac": achieved / fp64, "fp64_peak_tflops": fp64,
        "families_ms_per_step": {k: v[0] / args.steps for k, v in fam.items()},
        "hbm_peak_gbs": peaks.get("hbm_gbs"),
    }
    P.close()
    extra = None
    if not args.no_extra:
        try:
            extra = extra_workloads(args, torch, ft)
        except Exception as exc:
            extra = {"error": repr(exc)[:300]}
    cpu = None
    parity = None
    if world == 1 and not args.no_cpu:
        import tempfile
        ref_path = os.path.join(tempfile.mkdtemp(prefix="ftb200_"), "ref_fwd_field0.npy")
        try:
            threads, _ = host_cpu()
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
            out = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-sample", "--n", str(args.n),
                                  "--ref-out", ref_path], capture_output=True, text=True, timeout=900, env=env)
            cpu = json.loads(out.stdout.strip().splitlines()[-1])
        except Exception as exc:  # the line still carries the GPU numbers
            cpu = {"value": None, "error": repr(exc)[:200]}
        spin_cpu = cpu.pop("spin_s2", None) if isinstance(cpu, dict) else None
        spin_key = "spin_s2_n%d" % args.n
        if spin_cpu and isinstance(extra, dict) and spin_key in extra:
            extra[spin_key]["reference_cpu"] = spin_cpu
            extra[spin_key]["gpu_over_reference_cpu"] = extra[spin_key]["coeffs_per_s"] / spin_cpu["value"]
        if os.path.exists(ref_path):
            # the compiled reference's forward 'N' of field 0 (seed 20261203) against the GPU's:
            # the plain FP64 path (bit-identical to the single-field drop-in) and the mixed path
            ref = np.load(ref_path).ravel(order="F")
            os.remove(ref_path)
            nr, ni = np.linalg.norm(ref), np.abs(ref).max()
            parity = {"reference": "compiled reference ft_execute_sph2fourier('N'), field 0, on the host",
                      "plain_fp64_eps2": float(np.linalg.norm(fp64_f0 - ref) / nr),
                      "plain_fp64_epsinf": float(np.abs(fp64_f0 - ref).max() / ni),
                      "mixed_bf16_eps2": float(np.linalg.norm(mixed_f0 - ref) / nr),
                      "mixed_bf16_epsinf": float(np.abs(mixed_f0 - ref).max() / ni)}
            qpath = ref_path + ".quad.npy"
            if os.path.exists(qpath):
                # every form's forward of field 0 against the __float128 oracle on quad_cols(M)
                # columns (the compiled reference's own error beside them)
                hi = np.load(qpath)
                os.remove(qpath)
                cols = quad_cols(M)
                nh, ih = np.linalg.norm(hi), np.abs(hi).max()
                err = lambda x: {"eps2": float(np.linalg.norm(x - hi) / nh), "epsinf": float(np.abs(x - hi).max() / ih)}
                colsof = lambda flat: flat.reshape((n, M), order="F")[:, cols]
                pq = {"oracle": f"oracle/ft_quad.c (__float128 sweeps and connection multiply), {len(cols)} columns "
                                f"of every class over all orders, field 0 (seed {SEED})",
                      "reference": err(colsof(ref)), "plain_fp64": err(colsof(fp64_f0)), "mixed_bf16": err(colsof(mixed_f0))}
                for name, x in ((extra or {}).get("_field0_cols") or {}).items():
                    pq["shared_" + name] = err(x)
                parity["vs_quad"] = pq
            del ref
        fam_cpu = cpu.pop("families", None) if isinstance(cpu, dict) else None
        for key, v in (fam_cpu or {}).items():
            if isinstance(extra, dict) and isinstance(v, dict) and key in extra and "coeffs_per_s" in extra[key]:
                v["cores"] = cpu.get("cores")
                v["sample"] = "the compiled reference, one timed fwd+bwd 'N' after one warm-up, same size"
                extra[key]["reference_cpu"] = v
                extra[key]["gpu_over_reference_cpu"] = extra[key]["coeffs_per_s"] / v["value"]
    if isinstance(extra, dict):
        extra.pop("_field0_cols", None)   # host copies for the quad check, not part of the line
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 slices in the blocked sweeps, s8 digits in the connection multiply; exact f32 / s32 accumulation (f64 in and out)",
        "data": "synthetic: seeded U(-1,1) in the sph triangular layout (splitmix64, seed 20261203 + field)",
        "config": {"workload": f"batched mixed-precision sph2fourier+fourier2sph: {nf} fields of degree {n - 1} "
                               f"(n={n}, M={M}) sharing one plan, MIXED_BF16, per GPU",
                   "n": n, "M": M, "fields_per_gpu": nf, "precision": "MIXED_BF16", "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2: {nf} fields x {bytes_mat / 1e6:.0f} MB"},
        "vs_plain_fp64": {"plain_fp64_value": plain_value, "plain_fp64_ms_per_step": pms / psteps,
                          "ratio": value / plain_value, "plain": "FT_B200_FP64 direct sweeps + DMMA trmm, same fields"},
        "accuracy": {"fwd_eps2_vs_fp64": eps2, "fwd_epsinf_vs_fp64": epsinf, "roundtrip_eps2": rt2,
                     "roundtrip_epsinf": rtinf, "device_status": status,
                     "reference": "FT_B200_FP64 output (matches the oracle to 1e-14)"},
        "parity_vs_reference": parity,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nf * bytes_mat, "d2h_bytes_per_step": nf * bytes_mat,
                "api": "ft_b200_execute_shared_host (forward 'N' then backward 'N' on page-locked host fields; copies "
                       "of one group of fields overlap the transforms of the previous group)",
                "steps": e2e_steps, "host_group": int(os.environ.get("FT_B200_HOST_GROUP", "4"))},
        "gpu_launches": launches,
        "clocks": clocks,
        "workloads": extra,
    }
    print(json.dumps(line))


def plain_single(args, torch, ft):
    """Plain FP64 drop-in, one field of degree n - 1 (device-resident), with the FP64
    roofline of its dominant kernel family."""
    import numpy as np
    n = args.n
    M = 2 * n - 1
    A = ft.sphrand(n, SEED)
    P = ft.plan_sph2fourier(n)
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def step():
        ft.execute_dev(P, True, "N", d.data_ptr(), n, M, sptr)
        ft.execute_dev(P, False, "N", d.data_ptr(), n, M, sptr)
    step()
    back = d.cpu().numpy().reshape((n, M), order="F")
    eps2 = float(np.linalg.norm(back - A) / np.linalg.norm(A))
    epsinf = float(np.abs(back - A).max() / np.abs(A).max())
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    steps = max(5, args.steps // 2)
    ft.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    rot_ms, rot_n = ft.profile_read(0)
    trmm_ms, trmm_n = ft.profile_read(1)
    ft.profile(False)
    ms = e0.elapsed_time(e1)
    # end to end through the drop-in host API (pinned host array)
    hbuf = torch.empty(n * M, dtype=torch.float64, pin_memory=True)
    hbuf.copy_(torch.from_numpy(A.ravel(order="F")))
    Ah = hbuf.numpy().reshape((M, n)).T
    ft.execute_sph2fourier("N", P, Ah)
    ft.execute_fourier2sph("N", P, Ah)
    reps = 3 if n >= 2048 else 30   # a few ms per call at degree 1023: more calls for a steady mean
    t0 = time.perf_counter()
    for _ in range(reps):
        ft.execute_sph2fourier("N", P, Ah)
        ft.execute_fourier2sph("N", P, Ah)
    e2e = n * n * reps / (time.perf_counter() - t0)
    P.close()
    fp64 = fp64_peak_tflops(torch)
    rot_flops = 6 * rotations_sph(n)
    tr_flops = trmm_flops(n, M)
    famname = "rotations" if rot_ms >= trmm_ms else "trmm"
    per_launch = (rot_ms / max(rot_n, 1)) if famname == "rotations" else (trmm_ms / max(trmm_n, 1))
    flops = rot_flops if famname == "rotations" else tr_flops
    achieved = flops / (per_launch * 1e-3) / 1e12
    traffic = profiled_traffic(f"sph_n{n}", famname)
    total = 2 * (rot_flops + tr_flops)
    return {
        "coeffs_per_s": n * n * steps / (ms * 1e-3), "ms_per_step": ms / steps,
        "workload": f"plain FP64 sph2fourier+fourier2sph, degree {n - 1}, 1 field, device-resident plan",
        "roundtrip_eps2": eps2, "roundtrip_epsinf": epsinf,
        "e2e_coeffs_per_s": e2e, "e2e_api": "ft_execute_sph2fourier + ft_execute_fourier2sph on a pinned host array",
        "roofline": {"bound": "fp64", "kernel": "rot_kernel (Givens sweeps)" if famname == "rotations" else "gemm_tri_kernel (DMMA trmm)",
                     "achieved": achieved, "peak": fp64, "unit": "TFLOP/s", "frac": achieved / fp64, "traffic": traffic,
                     "peak_source": "measured in bench.py: cuBLAS DGEMM 8192^3 burst",
                     "flops_per_launch": flops, "ms_per_launch": per_launch,
                     "families_ms_per_step": {"rotations": rot_ms / steps, "trmm": trmm_ms / steps},
                     "step_fp64_frac": total / (ms / steps * 1e-3) / 1e12 / fp64}}


def profile_case(n: int, precision: str, fields: int) -> None:
    """Small fixed programs for ncu captures (no timing).  fp64: one field through the
    plain drop-in path, two forward transforms.  mixed / mixed4: `fields` fields sharing
    a plan through ft_b200_execute_shared_dev (MIXED_BF16 / MIXED_BF16X4), two forward
    transforms (the first builds the slice images)."""
    import torch
    import fasttransforms_b200 as ft
    M = 2 * n - 1
    P = ft.plan_sph2fourier(n)
    s = torch.cuda.current_stream().cuda_stream
    if precision == "fp64":
        d = [torch.from_numpy(ft.sphrand(n, SEED).ravel(order="F").copy()).cuda()]
        for _ in range(2):
            ft.execute_dev(P, True, "N", d[0].data_ptr(), n, M, s)
    else:
        prec = ft.MIXED_BF16 if precision == "mixed" else ft.MIXED_BF16X4
        d = [torch.from_numpy(ft.sphrand(n, SEED + f).ravel(order="F").copy()).cuda() for f in range(fields)]
        for _ in range(2):
            ft.execute_shared_dev(P, True, "N", [t.data_ptr() for t in d], prec, s)
    torch.cuda.synchronize()
    status = ft.device_status(P)
    P.close()
    print(json.dumps({"profile_case": f"sph n={n}, {precision}, {len(d)} field(s)", "device_status": status,
                      "max_abs": max(float(t.abs().max()) for t in d)}))


_FP64_PEAK = []


def _fp64_peak(torch) -> float:
    if not _FP64_PEAK:
        _FP64_PEAK.append(fp64_peak_tflops(torch))
    return _FP64_PEAK[0]


def _family_timing(torch, fwd, bwd, reps=5, breakdown=None):
    """Mean device time (ms) of fwd(); bwd() after one untimed pair, CUDA events on the stream.
    With a dict for breakdown: a second timed loop with the library's per-launch events on, whose
    per-step milliseconds of the rotation sweeps, the triangular multiplies and the other kernels
    go into it."""
    import fasttransforms_b200 as ft
    st = torch.cuda.current_stream()
    fwd(); bwd()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fwd(); bwd()
    e1.record(st)
    torch.cuda.synchronize()
    if breakdown is not None:
        ft.profile(True)
        for _ in range(reps):
            fwd(); bwd()
        torch.cuda.synchronize()
        for fam, key in ((0, "rotations"), (1, "trmm"), (2, "other")):
            ms, nl = ft.profile_read(fam)
            breakdown[key + "_ms"] = ms / reps
            breakdown[key + "_launches"] = nl / reps
        ft.profile(False)
    return e0.elapsed_time(e1) / reps


def _rotation_roofline(torch, out, brk, rotations_per_step):
    """The sweeps' FP64 rate (6 flops a rotation) from the profiled per-step time."""
    if brk.get("rotations_ms", 0) > 0:
        tf = 6.0 * rotations_per_step / (brk["rotations_ms"] * 1e-3) / 1e12
        out["rotation_sweeps"] = {"ms_per_step": brk["rotations_ms"], "rotations_per_step": int(rotations_per_step),
                                  "tflops": tf, "fp64_peak_tflops": _fp64_peak(torch), "frac": tf / _fp64_peak(torch),
                                  "breakdown_ms_per_step": brk}


def rotations_rect(n):
    """Rotations of one rectdisk hi2lo: order m (column m, m = 2 .. n - 1), sweeps j = m - 2, .., m mod 2,
    n - 2 - j rotations each (src/rotations/rotations_default.c:73-78)."""
    import numpy as np
    j = np.arange(0, max(n - 2, 0), dtype=np.int64)
    c = np.maximum(0, (n - 1 - (j + 2)) // 2 + 1)
    return int(np.sum(c * np.maximum(0, n - 2 - j)))


def rotations_disk(n, M):
    """Rotations of one disk hi2lo (both columns of each order m = 2 .. M/2; sweeps j = m - 2, .., m mod 2,
    n - 1 - (j + 1) / 2 rotations each; src/rotations/rotations_default.c:59-64)."""
    import numpy as np
    j = np.arange(0, max(M // 2 - 1, 0), dtype=np.int64)
    c = np.maximum(0, (M // 2 - (j + 2)) // 2 + 1)
    return int(2 * np.sum(c * np.maximum(0, n - 1 - (j + 1) // 2)))


def rotations_tet(n, slabs=True):
    """Element rotations of one tetrahedral hi2lo with L = M = n: the triangle sweeps of order o on o + 1
    columns (o < n), sum over j < o of n - 1 - j each; with slabs, also per slab m the sweeps j < m
    across the slab, n - 1 - j column pairs of n elements each (src/drivers.c:510-528)."""
    import numpy as np
    o = np.arange(n, dtype=np.int64)
    tri = np.sum((o + 1) * (o * (n - 1) - o * (o - 1) // 2))
    m = np.arange(n, dtype=np.int64)
    tet = np.sum((m * (n - 1) - m * (m - 1) // 2) * n) if slabs else 0
    return int(tri + tet)


def family_rectdisk(n):
    import numpy as np
    import torch
    import fasttransforms_b200 as ft
    sp = torch.cuda.current_stream().cuda_stream
    P = ft.plan_rectdisk2cheb(n, 0.0)
    A = ft.rectdiskrand(n, SEED)
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    f = lambda: ft.execute_dev(P, True, "N", d.data_ptr(), n, n, sp)
    b = lambda: ft.execute_dev(P, False, "N", d.data_ptr(), n, n, sp)
    d.copy_(torch.from_numpy(A.ravel(order="F").copy()))
    f(); b()
    torch.cuda.synchronize()
    rt = float(np.linalg.norm(d.cpu().numpy() - A.ravel(order="F")) / np.linalg.norm(A))
    brk = {}
    ms = _family_timing(torch, f, b, breakdown=brk)
    P.close()
    coeffs = n * (n + 1) // 2
    out = {"coeffs_per_s": coeffs / (ms * 1e-3), "ms_per_step": ms, "roundtrip_eps2": rt,
           "workload": f"rectdisk2cheb + cheb2rectdisk 'N', beta = 0, degree {n - 1}, 1 field {n} x {n} (plain FP64; "
                       f"{coeffs} coefficients)"}
    _rotation_roofline(torch, out, brk, 2 * rotations_rect(n))
    return out


def family_ann(n):
    import numpy as np
    import torch
    import fasttransforms_b200 as ft
    sp = torch.cuda.current_stream().cuda_stream
    rho = float(np.sqrt(1 / 3))
    P = ft.plan_ann2cxf(n, 0.0, 0.0, 0.0, rho)
    A = ft.diskrand(n, SEED)
    M = A.shape[1]
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    f = lambda: ft.execute_dev(P, True, "N", d.data_ptr(), n, M, sp)
    b = lambda: ft.execute_dev(P, False, "N", d.data_ptr(), n, M, sp)
    f(); b()
    torch.cuda.synchronize()
    rt = float(np.linalg.norm(d.cpu().numpy() - A.ravel(order="F")) / np.linalg.norm(A))
    brk = {}
    ms = _family_timing(torch, f, b, breakdown=brk)
    P.close()
    coeffs = 2 * n * n - n
    out = {"coeffs_per_s": coeffs / (ms * 1e-3), "ms_per_step": ms, "roundtrip_eps2": rt,
           "workload": f"ann2cxf + cxf2ann 'N', alpha = beta = 0, rho = sqrt(1/3), degree {n - 1}, 1 field {n} x {M} "
                       f"(plain FP64)"}
    _rotation_roofline(torch, out, brk, 2 * rotations_disk(n, M))
    return out


def family_tet(n):
    import numpy as np
    import torch
    import fasttransforms_b200 as ft
    sp = torch.cuda.current_stream().cuda_stream
    P = ft.plan_tet2cheb(n, 0.0, 0.0, 0.0, 0.0)
    A = ft.tetrand(n, SEED)
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    f = lambda: ft.execute_tet_dev(P, True, "N", d.data_ptr(), n, n, n, sp)
    b = lambda: ft.execute_tet_dev(P, False, "N", d.data_ptr(), n, n, n, sp)
    f(); b()
    torch.cuda.synchronize()
    rt = float(np.linalg.norm(d.cpu().numpy() - A.ravel(order="F")) / np.linalg.norm(A))
    brk = {}
    ms = _family_timing(torch, f, b, breakdown=brk)
    P.close()
    coeffs = n * (n + 1) * (n + 2) // 6
    out = {"coeffs_per_s": coeffs / (ms * 1e-3), "ms_per_step": ms, "roundtrip_eps2": rt,
           "workload": f"tet2cheb + cheb2tet 'N', parameters 0, degree {n - 1}, 1 field {n} x {n} x {n} (plain FP64; "
                       f"{coeffs} coefficients)",
           "note": "rotation_sweeps: the triangle sweeps down the columns (the rotation kernel); the sweeps across "
                   "the slabs are not in the profiled families"}
    _rotation_roofline(torch, out, brk, 2 * rotations_tet(n, slabs=False))
    return out


def family_grid(kind, n):
    """The family's full transform on the device: to Chebyshev / Fourier, synthesis, analysis, back."""
    import numpy as np
    import torch
    import fasttransforms_b200 as ft
    sp = torch.cuda.current_stream().cuda_stream
    if kind == "disk":
        P, PS, PA, grid = ft.plan_disk2cxf(n, 0.0, 0.0), ft.plan_disk_synthesis(n), ft.plan_disk_analysis(n), ft.execute_disk_grid_dev
        coeffs = 2 * n * n - n
    elif kind == "annulus":
        rho = float(np.sqrt(1 / 3))
        P, PS, PA = ft.plan_ann2cxf(n, 0.0, 0.0, 0.0, rho), ft.plan_annulus_synthesis(n, rho), ft.plan_annulus_analysis(n, rho)
        grid = ft.execute_annulus_grid_dev
        coeffs = 2 * n * n - n
    elif kind == "rectdisk":
        P, PS, PA = ft.plan_rectdisk2cheb(n, 0.0), ft.plan_rectdisk_synthesis(n), ft.plan_rectdisk_analysis(n)
        grid = ft.execute_rectdisk_grid_dev
        coeffs = n * (n + 1) // 2
    else:
        P, PS, PA, grid = ft.plan_tri2cheb(n, 0.0, 0.0, 0.0), ft.plan_tri_synthesis(n), ft.plan_tri_analysis(n), ft.execute_tri_grid_dev
        coeffs = n * (n + 1) // 2
    A = ft.rand_layout({"annulus": "disk", "rectdisk": "rect"}.get(kind, kind), n, SEED)
    M = A.shape[1]
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    p = d.data_ptr()
    f = lambda: (ft.execute_dev(P, True, "N", p, n, M, sp), grid(PS, False, "N", p, n, M, sp))
    b = lambda: (grid(PA, True, "N", p, n, M, sp), ft.execute_dev(P, False, "N", p, n, M, sp))
    f(); b()
    torch.cuda.synchronize()
    rt = float(np.linalg.norm(d.cpu().numpy() - A.ravel(order="F")) / np.linalg.norm(A))
    ms = _family_timing(torch, f, b)
    ms_grid = _family_timing(torch, lambda: grid(PS, False, "N", p, n, M, sp), lambda: grid(PA, True, "N", p, n, M, sp))
    for q in (P, PS, PA):
        q.close()
    return {"coeffs_per_s": coeffs / (ms * 1e-3), "ms_per_step": ms, "grid_synthesis_plus_analysis_ms": ms_grid,
            "roundtrip_eps2": rt,
            "workload": f"{kind}: to the Chebyshev / Fourier series, synthesis on the grid, analysis, back ('N'), "
                        f"degree {n - 1}, 1 field {n} x {M} (plain FP64, cuFFT DFTs inside the grid stage)"}


def family_tet_grid(n):
    """tet2cheb + synthesis on the n^3 grid, analysis + cheb2tet ('N'), on the device."""
    import numpy as np
    import torch
    import fasttransforms_b200 as ft
    sp = torch.cuda.current_stream().cuda_stream
    P, TS, TA = ft.plan_tet2cheb(n, 0.0, 0.0, 0.0, 0.0), ft.plan_tet_synthesis(n), ft.plan_tet_analysis(n)
    A = ft.tetrand(n, SEED)
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    p = d.data_ptr()
    f = lambda: (ft.execute_tet_dev(P, True, "N", p, n, n, n, sp), ft.execute_tet_grid_dev(TS, False, "N", p, n, n, n, sp))
    b = lambda: (ft.execute_tet_grid_dev(TA, True, "N", p, n, n, n, sp), ft.execute_tet_dev(P, False, "N", p, n, n, n, sp))
    f(); b()
    torch.cuda.synchronize()
    rt = float(np.linalg.norm(d.cpu().numpy() - A.ravel(order="F")) / np.linalg.norm(A))
    ms = _family_timing(torch, f, b)
    ms_grid = _family_timing(torch, lambda: ft.execute_tet_grid_dev(TS, False, "N", p, n, n, n, sp),
                             lambda: ft.execute_tet_grid_dev(TA, True, "N", p, n, n, n, sp))
    for q in (P, TS, TA):
        q.close()
    coeffs = n * (n + 1) * (n + 2) // 6
    return {"coeffs_per_s": coeffs / (ms * 1e-3), "ms_per_step": ms, "grid_synthesis_plus_analysis_ms": ms_grid,
            "roundtrip_eps2": rt,
            "workload": f"tet: tet2cheb, synthesis on the {n}^3 grid, analysis, cheb2tet ('N'), degree {n - 1}, 1 field "
                        f"(plain FP64, cuFFT DFTs inside the grid stage)"}


def extra_workloads(args, torch, ft):
    """Secondary workloads (reported beside the headline, same device timing rules)."""
    import numpy as np
    out = {"plain_fp64_n%d" % args.n: plain_single(args, torch, ft)}
    if args.n != 1024:   # the plain path's other degree, 1023 (its 16.8 MB matrix stays in L2)
        a2 = argparse.Namespace(**vars(args))
        a2.n = 1024
        out["plain_fp64_n1024"] = plain_single(a2, torch, ft)
        out["plain_fp64_n1024"]["note"] = "matrix (16.8 MB) resident in L2 between steps"
    st = torch.cuda.current_stream()
    sp = st.cuda_stream

    def timed(fn, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    # the full spherical-harmonic transform on the device: sph2fourier + grid synthesis, then
    # grid analysis + fourier2sph (plain FP64), one field of degree n - 1
    n = args.n
    M = 2 * n - 1
    Pn, PS, PA = ft.plan_sph2fourier(n), ft.plan_sph_synthesis(n), ft.plan_sph_analysis(n)
    A = ft.sphrand(n, SEED)
    d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    dp = d.data_ptr()

    def sht():
        ft.execute_dev(Pn, True, "N", dp, n, M, sp)
        ft.execute_sph_grid_dev(PS, "sph_synthesis", "N", dp, n, M, sp)
        ft.execute_sph_grid_dev(PA, "sph_analysis", "N", dp, n, M, sp)
        ft.execute_dev(Pn, False, "N", dp, n, M, sp)

    def grid_only():
        ft.execute_sph_grid_dev(PS, "sph_synthesis", "N", dp, n, M, sp)
        ft.execute_sph_grid_dev(PA, "sph_analysis", "N", dp, n, M, sp)
    sht()
    back = d.cpu().numpy().reshape((n, M), order="F")
    rt = float(np.linalg.norm(back - A) / np.linalg.norm(A))
    for _ in range(max(1, args.warmup)):
        sht()
    ms = timed(sht, max(3, args.steps // 4))
    ms_grid = timed(grid_only, max(3, args.steps // 4))
    out["sht_full_n%d" % n] = {"coeffs_per_s": n * n / (ms * 1e-3), "ms_per_step": ms,
                              "grid_synthesis_plus_analysis_ms": ms_grid, "roundtrip_eps2": rt,
                              "workload": f"sph2fourier + synthesis, analysis + fourier2sph, degree {n - 1}, 1 field, "
                                          f"{n} x {M} grid (plain FP64, cuFFT DFTs inside the grid stage)"}
    del d
    for q in (Pn, PS, PA):
        q.close()
    # spin-weighted transform (s = 2): spinsph2fourier + fourier2spinsph 'N' on one complex
    # field of degree n - 1 (plain FP64), and its rotation stage alone (hi2lo + lo2hi)
    s = 2
    SP, SRP = ft.plan_spinsph2fourier(n, s), ft.plan_rotspinsphere(n, s)
    Z = ft.spinsphrand(n, s, SEED)
    dz = torch.from_numpy(Z.ravel(order="F").view(np.float64).copy()).cuda()
    zp = dz.data_ptr()

    def spin():
        ft.execute_spin_dev(SP, True, "N", zp, n, M, sp)
        ft.execute_spin_dev(SP, False, "N", zp, n, M, sp)

    def spin_rot():
        ft.spin_rotations_dev(SRP, True, zp, M, sp)
        ft.spin_rotations_dev(SRP, False, zp, M, sp)
    spin()
    back = dz.cpu().numpy().view(np.complex128).reshape((n, M), order="F")
    rt = float(np.linalg.norm(back - Z) / np.linalg.norm(Z))
    for _ in range(max(1, args.warmup)):
        spin()
    ms = timed(spin, max(3, args.steps // 4))
    ms_rot = timed(spin_rot, max(3, args.steps // 4))
    out["spin_s2_n%d" % n] = {"coeffs_per_s": n * n / (ms * 1e-3), "ms_per_step": ms,
                             "rotations_hi2lo_plus_lo2hi_ms": ms_rot, "roundtrip_eps2": rt,
                             "workload": f"spinsph2fourier + fourier2spinsph 'N', s = {s}, degree {n - 1}, "
                                         f"1 complex field {n} x {M} (plain FP64)"}
    del dz
    SP.close()
    SRP.close()
    # the other families' drop-in transforms and the disk / triangle grids, one field each, fwd+bwd
    # 'N' on the device (plain FP64); each in its own guard so that one failure leaves the rest
    for name, fn in (("rectdisk_n4096", lambda: family_rectdisk(4096)), ("ann_n2048", lambda: family_ann(2048)),
                     ("tet_n256", lambda: family_tet(256)), ("disk_full_grid_n2048", lambda: family_grid("disk", 2048)),
                     ("tri_full_grid_n2048", lambda: family_grid("tri", 2048)),
                     ("annulus_full_grid_n2048", lambda: family_grid("annulus", 2048)),
                     ("rectdisk_full_grid_n2048", lambda: family_grid("rectdisk", 2048)),
                     ("tet_full_grid_n128", lambda: family_tet_grid(128))):
        try:
            out[name] = fn()
        except Exception as exc:
            out[name] = {"error": repr(exc)[:200]}
    # 64 FP64 sph fields, degrees drawn from {127, 255, 511, 1023, 2047}, one launch per stage,
    # fwd+bwd captured in one CUDA graph
    rng = np.random.default_rng(SEED)
    degs = [int(d) + 1 for d in rng.choice([127, 255, 511, 1023, 2047], size=64)]
    plans = {n: ft.plan_sph2fourier(n) for n in sorted(set(degs))}
    P = [plans[n] for n in degs]
    Ns = [p.n for p in P]
    Ms = [p.M for p in P]
    data = [torch.from_numpy(ft.sphrand(n, SEED + f).ravel(order="F").copy()).cuda() for f, n in enumerate(degs)]
    ptrs = [d.data_ptr() for d in data]
    side = torch.cuda.Stream()
    side.wait_stream(st)
    with torch.cuda.stream(side):
        for _ in range(max(1, args.warmup)):
            ft.execute_batched_dev(P, True, "N", ptrs, Ns, Ms, side.cuda_stream)
            ft.execute_batched_dev(P, False, "N", ptrs, Ns, Ms, side.cuda_stream)
    st.wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cs = torch.cuda.current_stream().cuda_stream
        ft.execute_batched_dev(P, True, "N", ptrs, Ns, Ms, cs)
        ft.execute_batched_dev(P, False, "N", ptrs, Ns, Ms, cs)
    ms = timed(g.replay, max(3, args.steps // 2))
    coeffs = sum(n * n for n in degs)
    # same fields one plan call after another, eager, for comparison
    loop = lambda: [ft.execute_dev(p, fw, "N", d.data_ptr(), p.n, p.M, sp) for fw in (True, False) for p, d in zip(P, data)]
    loop()   # first calls per degree build task lists and tune launch shapes
    ms_loop = timed(loop, max(3, args.steps // 4))
    out["batched_uneven_64"] = {"coeffs_per_s": coeffs / (ms * 1e-3), "ms_per_step": ms,
                                "per_field_loop_coeffs_per_s": coeffs / (ms_loop * 1e-3),
                                "degrees": "64 fields, U{127,255,511,1023,2047} seed 20261203",
                                "graph": "fwd+bwd captured in one CUDA graph"}
    del g, data
    for p in plans.values():
        p.close()
    # 16 fields of degree 4095 sharing one plan: every precision of ft_b200_execute_shared_dev
    n = 4096
    Pn = ft.plan_sph2fourier(n)
    M = Pn.M
    fields = [torch.from_numpy(ft.sphrand(n, SEED + f).ravel(order="F").copy()).cuda() for f in range(16)]
    fptr = [f.data_ptr() for f in fields]
    res = {}
    ref_out = None
    qcols = quad_cols(M)
    out["_field0_cols"] = {}
    field0 = fields[0].clone()   # the fields below are transformed in place; errors start from this copy
    for name, prec in (("fp64_direct", ft.FP64), ("fp64_blocked", ft.FP64_BLOCKED), ("mixed_bf16_3slices", ft.MIXED_BF16),
                       ("mixed_bf16_4slices", ft.MIXED_BF16X4)):
        x0 = field0.clone()
        ft.execute_shared_dev(Pn, True, "N", [x0.data_ptr()], prec, sp)   # builds tables outside timing
        torch.cuda.synchronize()
        out["_field0_cols"][name] = x0.view(M, n).t()[:, qcols].cpu().numpy()
        if ref_out is None:
            ref_out = x0
            err = 0.0
        else:
            err = float(torch.linalg.norm(x0 - ref_out) / torch.linalg.norm(ref_out))

        def step(prec=prec):
            ft.execute_shared_dev(Pn, True, "N", fptr, prec, sp)
            ft.execute_shared_dev(Pn, False, "N", fptr, prec, sp)
        step()
        ms = timed(step, 3)
        res[name] = {"coeffs_per_s": 16 * n * n / (ms * 1e-3), "ms_per_step": ms,
                     "eps2_fwd_vs_fp64_direct": err, "fields": "seeds 20261203 + f (field 0 for the error)"}
    out["shared_16_n4096"] = res
    del fields
    Pn.close()
    # sibling families at degree 2047, 8 fields per transform: the plain FP64 form (batched
    # path) and the shared-plan forms, with the forward errors of the mixed forms against
    # the FP64 transform of field 0
    for name, kind, params in (("tri_000", "tri", (0.0, 0.0, 0.0)), ("tri_hhh", "tri", (-0.5, -0.5, -0.5)),
                               ("disk_00", "disk", (0.0, 0.0))):
        n = 2048
        planner = ft.plan_tri2cheb if kind == "tri" else ft.plan_disk2cxf
        p = planner(n, *params)
        M = p.M
        fields = [torch.from_numpy(ft.rand_layout(kind, n, SEED + f).ravel(order="F").copy()).cuda() for f in range(8)]
        fptr = [f.data_ptr() for f in fields]
        field0 = fields[0].clone()
        per_field = n * (n + 1) // 2 if kind == "tri" else 2 * n * n - n

        def step():
            ft.execute_batched_dev([p] * 8, True, "N", fptr, [n] * 8, [M] * 8, sp)
            ft.execute_batched_dev([p] * 8, False, "N", fptr, [n] * 8, [M] * 8, sp)
        for _ in range(max(1, args.warmup)):
            step()
        ms = timed(step, max(3, args.steps // 4))
        res = {"coeffs_per_s": 8 * per_field / (ms * 1e-3), "ms_per_step": ms,
               "workload": f"{kind}{params}, degree {n - 1}, 8 fields, fwd+bwd 'N'"}
        ref_out = None
        for pname, prec in (("fp64_shared", ft.FP64), ("fp64_blocked", ft.FP64_BLOCKED),
                            ("mixed_bf16_3slices", ft.MIXED_BF16), ("mixed_bf16_4slices", ft.MIXED_BF16X4)):
            x0 = field0.clone()
            ft.execute_shared_dev(p, True, "N", [x0.data_ptr()], prec, sp)   # builds tables outside timing
            torch.cuda.synchronize()
            if ref_out is None:
                ref_out = x0
                e2 = einf = 0.0
            else:
                e2 = float(torch.linalg.norm(x0 - ref_out) / torch.linalg.norm(ref_out))
                einf = float((x0 - ref_out).abs().max() / ref_out.abs().max())

            def sstep(prec=prec):
                ft.execute_shared_dev(p, True, "N", fptr, prec, sp)
                ft.execute_shared_dev(p, False, "N", fptr, prec, sp)
            sstep()
            ms = timed(sstep, max(3, args.steps // 4))
            res[pname] = {"coeffs_per_s": 8 * per_field / (ms * 1e-3), "ms_per_step": ms,
                          "eps2_fwd_vs_fp64": e2, "epsinf_fwd_vs_fp64": einf}
        res["mixed_bf16_over_fp64"] = res["mixed_bf16_3slices"]["coeffs_per_s"] / res["coeffs_per_s"]
        out[name] = res
        del fields, field0, ref_out
        p.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--fields", type=int, default=16, help="fields sharing one plan in the headline workload")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--cpu-sample", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--ref-out", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--profile-case", action="store_true",
                    help="run one plan and two forward transforms (for ncu), no timing")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "mixed4"],
                    help="--profile-case path: plain FP64 (one field) or the shared-plan tensor-core paths")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.n, args.precision, args.fields)
        return
    if args.cpu_sample:
        print(json.dumps(cpu_sample(args.n, args.ref_out)))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
