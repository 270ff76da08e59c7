#!/usr/bin/env python
"""Benchmark: f128 GEMM GFLOP/s on one B200 (chosen Ozaki-II int8 path vs the
plain CUDA-core dd path), plus the CPU baseline and an end-to-end number.

Workload: C = A * B, m = n = k = 2048, full double-double entries (SplitMix64
seed 0, hi ~ U[-1,1), lo = hi * 2^-53 * U[-1,1)). One step = one GEMM.
  value  = chosen-path GFLOP/s (2mnk per step) with inputs resident in HBM,
           device-timed with CUDA events; L2 flushed between timed steps.
  e2e    = the same GEMM through the host-pointer C ABI (hp_f128_gemm) from
           pinned host buffers, copies inside the timed region.
Multi-GPU (torchrun): every rank runs its own independent GEMM (weak scaling,
no collective in the data path); value = all ranks' flops / max rank time.

--impl reference times the reference algorithm on the host cores (the C++
restatement in oracle/, since the Rust reference cannot be built here) on a
bounded sample of C rows per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

M = N = K = 2048
# DRAM bytes (read + write) of one i8_gemm_pair_kernel launch at this size,
# from an ncu capture of `bench.py --profile-case gemm` (251.8 MB read: every
# residue plane once; 100.3 MB written, the rest of the 125.8 MB of product
# residues still in L2 when the kernel ends).
I8_GEMM_TRAFFIC_BYTES = 352043776
METRIC = "f128 GEMM GFLOP/s; SPD solves/s at ≤1e-25 rel err: chosen vs plain, 1 B200"
WORKLOAD = "f128 GEMM C=A*B, m=n=k=2048, full double-double entries (SplitMix64 seed 0)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons sampled DURING a timed region.

    NVML is polled every `period_s` seconds from a thread (the timed CUDA
    work releases the GIL in its driver calls), so that even a region of a
    few milliseconds gets several samples. The device is the CUDA device
    `index` of this process, found in NVML by its UUID (NVML numbers every
    GPU of the machine, CUDA only the visible ones). Falls back to polling
    nvidia-smi (every 200 ms) when NVML is unavailable.
    """
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, index: int, period_s: float = 0.002):
        self.index = index
        self.period = period_s
        self.rows = []
        self.proc = None
        self.th = None
        self.nvml = None
        self.stop_evt = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = getattr(torch.cuda.get_device_properties(self.index), "uuid", None)
        if uuid is not None:
            u = str(uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
        except Exception:
            self.nvml = None
        if self.nvml is not None:
            self.th = threading.Thread(target=self._poll, daemon=True)
            self.th.start()
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _poll(self):
        nv, h = self.nvml
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_evt.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), bits))
            except Exception:
                pass
            time.sleep(self.period)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.nvml is not None:
            self.stop_evt.set()
            self.th.join(timeout=2)
            sm = [r[0] for r in self.rows]
            reasons = sorted({k for r in self.rows for k, bit in self.REASONS.items() if r[2] & bit})
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": max(r[1] for r in self.rows) if self.rows else None,
                    "reasons": reasons, "samples": len(self.rows), "source": f"NVML every {self.period * 1e3:g} ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": "nvidia-smi every 200 ms"}


# ---------------------------------------------------------------- helpers
def init_dist(backend: str = "nccl"):
    """(world, rank, local_rank, dist or None) from the launcher's environment;
    one process per GPU, rendezvous on MASTER_ADDR (127.0.0.1 for this
    launcher). A short timeout makes ranks that wait for a missing peer fail."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return world, rank, local, None
    import datetime

    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local, dist


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of the ranks' values (times are reported as the slowest
    rank's); x itself when running on one process."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def cpu_sample_gflops(target_s: float = 12.0, threads: int | None = None) -> dict:
    """Oracle (C++ restatement of linalg.rs:150 gemm) on a bounded row sample,
    on all host threads or on `threads`."""
    import numpy as np

    import oracle
    from quadprec_b200.workloads import gemm_operands

    a, b = gemm_operands(M, N, K, seed=0)
    prev = oracle.num_threads()
    if threads is not None:
        oracle.set_threads(threads)
    threads = oracle.num_threads()
    rows = max(1, threads)
    t0 = time.perf_counter()
    oracle.gemm(a, b, M, N, K, rows=(0, rows))
    dt = time.perf_counter() - t0
    reps = max(1, min(64, int(target_s / max(dt, 1e-3))))
    total_rows = 0
    t0 = time.perf_counter()
    for r in range(reps):
        r0 = (r * rows) % M
        oracle.gemm(a, b, M, N, K, rows=(r0, min(M, r0 + rows)))
        total_rows += min(M, r0 + rows) - r0
    dt = time.perf_counter() - t0
    oracle.set_threads(prev)
    return {"value": 2.0 * total_rows * N * K / dt / 1e9, "unit": "GFLOP/s", "cores": threads, "kind": "port",
            "sample": f"{total_rows} of {M} rows of C (each a full 2048x2048 dd dot-product sweep), "
                      f"{dt:.1f} s; oracle/hp_oracle.cpp restates crates/quad/src/linalg.rs:150-165"}


def run_reference(args):
    """--impl reference: the reference algorithm on host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    from quadprec_b200.workloads import gemm_operands

    a, b = gemm_operands(M, N, K, seed=0)
    threads = oracle.num_threads()
    rows = threads
    for w in range(args.warmup):
        oracle.gemm(a, b, M, N, K, rows=(0, rows))
    t0 = time.perf_counter()
    done = 0
    for s in range(args.steps):
        r0 = (s * rows) % M
        oracle.gemm(a, b, M, N, K, rows=(r0, r0 + rows))
        done += rows
    dt = time.perf_counter() - t0
    v = 2.0 * done * N * K / dt / 1e9
    line = {"metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (double-double EFT arithmetic)",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "m": M, "n": N, "k": K,
                       "step": f"{rows} rows of C per step (bounded sample of the 2048^3 GEMM)"},
            "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "port",
                             "sample": f"{done} rows of C over {args.steps} steps; C++ restatement of "
                                       "crates/quad/src/linalg.rs:150-165 (no Rust toolchain on this image)"},
            "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def profile_case(args):
    """Chosen-path GEMM steps only: the command that ncu captures."""
    import torch

    import quadprec_b200 as hp
    from quadprec_b200.workloads import gemm_operands

    a_np, b_np = gemm_operands(M, N, K, seed=0)
    A = torch.from_numpy(a_np).cuda()
    B = torch.from_numpy(b_np).cuda()
    C = torch.empty((M, N, 2), dtype=torch.float64, device="cuda")
    sptr = torch.cuda.current_stream().cuda_stream
    for _ in range(args.warmup + args.steps):
        hp.f128_gemm_dev(A, B, C, M, N, K, hp.OZAKI, stream=sptr)
    torch.cuda.synchronize()
    print("profile case done", file=sys.stderr)
    return 0


def gemm_f512_fixture():
    """f512 values of sampled entries of the benchmark GEMMs (seed-0 operands),
    generated by tests/golden/make_gemm_f512_fixture.py; None if absent."""
    import numpy as np

    p = os.path.join(REPO, "tests", "golden", "gemm_f512_sample.npz")
    return np.load(p) if os.path.exists(p) else None


def f512_errors(c, a, b, name, atb=False):
    """Normwise error of C over the fixture's sampled entries (4096 random +
    rows 0 and m-1) against the f512 oracle: || |A||B| ||-relative and ||C*||-relative."""
    from quadprec_b200.workloads import sample_abs_products, sample_index, sampled_error

    fx = gemm_f512_fixture()
    if fx is None or name not in fx:
        return None
    m = c.shape[0]
    idx = sample_index(m, c.shape[1])
    e_ab, e_c = sampled_error(c, fx[name], sample_abs_products(a, b, idx, atb), idx)
    return {"normwise_vs_absAB": e_ab, "normwise_vs_C": e_c, "entries": int(len(idx))}


def gemm_more_section(hp, torch, dev, stream, sptr, world, dist):
    """gemm_atb at 2048^3 (f128) and mf_gemm at 1024^3 (f256), chosen and plain,
    each with its error against the f512 oracle on sampled entries."""
    from quadprec_b200.workloads import dd_to_qd, gemm_operands

    def timed(fn, steps):
        fn()
        torch.cuda.synchronize()
        s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(steps):
            fn()
        e0.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(s0.elapsed_time(e0) / steps, dist, dev)

    out = {}
    a, b = gemm_operands(M, N, K, seed=0, atb=True)
    A, B = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    C = torch.empty((M, N, 2), dtype=torch.float64, device=dev)
    sec = out.setdefault("f128_gemm_atb_2048", {"unit": "GFLOP/s (2mnk f128 ops)"})
    for name, mode, steps in (("chosen", hp.OZAKI, 5), ("plain", hp.PLAIN, 1)):
        ms = timed(lambda: hp.f128_gemm_dev(A, B, C, M, N, K, mode, atb=True, stream=sptr), steps)
        torch.cuda.synchronize()
        sec[name] = {"gflops": world * 2.0 * M * N * K / (ms * 1e-3) / 1e9, "ms": ms,
                     "err_vs_f512": f512_errors(C.cpu().numpy(), a, b, "f128_gemm_atb_2048", atb=True)}
    sec["chosen_over_plain"] = sec["plain"]["ms"] / sec["chosen"]["ms"]
    del A, B, C
    n4 = 1024
    a, b = gemm_operands(n4, n4, n4, seed=0)
    a4, b4 = dd_to_qd(a), dd_to_qd(b)  # limbs 2-3 zero (full double-double entries)
    A, B = torch.from_numpy(a4).to(dev), torch.from_numpy(b4).to(dev)
    C = torch.empty((n4, n4, 4), dtype=torch.float64, device=dev)
    sec = out.setdefault("f256_mf_gemm_1024", {"unit": "GFLOP/s (2mnk f256 ops)"})
    for name, mode, steps in (("chosen", hp.OZAKI, 5), ("plain", hp.PLAIN, 1)):
        ms = timed(lambda: hp.f256_gemm_dev(A, B, C, n4, n4, n4, mode, stream=sptr), steps)
        torch.cuda.synchronize()
        sec[name] = {"gflops": world * 2.0 * n4 ** 3 / (ms * 1e-3) / 1e9, "ms": ms,
                     "err_vs_f512": f512_errors(C.cpu().numpy(), a4, b4, "f256_gemm_1024")}
    sec["chosen_over_plain"] = sec["plain"]["ms"] / sec["chosen"]["ms"]
    return out


SPD_LATTICE = (5, 10, 10)  # 500 centres x 4 exponents = 2000 basis functions


def spd_section(hp, torch, dev, stream, sptr, args, rank, world, dist):
    """Overlap SPD solve to <= 1e-25: assemble S (f128, GPU) + factor + refine.

    One step = one complete solve of the n = 2000 overlap system (assembly of
    S from the basis on the device, Cholesky, refinement to max|dx| <= 1e-28
    max|x|). Reported as solves/s for the chosen (residue-domain tcgen05
    Cholesky) and plain (reference f128 Cholesky + f256 residuals) modes.
    """
    import ctypes

    import numpy as np

    from quadprec_b200.workloads import overlap_spd_problem

    cen, alpha, b = overlap_spd_problem(*SPD_LATTICE, seed=0)
    n = len(alpha)
    dcen = torch.from_numpy(np.ascontiguousarray(cen)).to(dev)
    dal = torch.from_numpy(alpha).to(dev)
    b2 = np.stack([b, np.zeros_like(b)], -1)
    db = torch.from_numpy(b2).to(dev)
    dS = torch.empty((n, n, 2), dtype=torch.float64, device=dev)
    dx = torch.empty((n, 2), dtype=torch.float64, device=dev)
    lib = hp.lib()
    fix = os.path.join(REPO, "tests", "golden", "overlap_5x10x10.npz")
    xs = np.load(fix)["x_star"] if os.path.exists(fix) else None

    def one(mode):
        info = hp.RefineInfo()
        pv = ctypes.c_int64(-1)
        hp.check(lib.hp_overlap_norm_dd_dev(n, dcen.data_ptr(), dal.data_ptr(), dS.data_ptr(), sptr))
        hp.check(lib.hp_spd_solve_refined_dev(dS.data_ptr(), db.data_ptr(), n, mode, 1e-28, 10, dx.data_ptr(),
                                              ctypes.byref(info), ctypes.byref(pv), sptr))
        return info

    out = {"workload": f"overlap SPD, {n} s-Gaussians on a jittered 5x10x10 lattice (spacing 1.4 bohr, 4 exponents "
                       "log-uniform in [0.01, 10]), b ~ N(0,1) (Irwin-Hall); S assembled in f128 on the GPU",
           "n": n, "unit": "solves/s", "target": "max rel err <= 1e-25 vs the f512 oracle solution"}
    for name, mode in (("chosen", hp.OZAKI), ("plain", hp.PLAIN)):
        one(mode)  # warm-up
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        evs, infos = [], []
        for _ in range(args.spd_steps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            infos.append(one(mode))
            e.record(stream)
            evs.append((s, e))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(z) for a, z in evs) / args.spd_steps
        ms = max_over_ranks(ms, dist, dev)
        x = dx.cpu().numpy()
        err = None
        if xs is not None:
            d = (xs[:, 0] - x[:, 0]) + (xs[:, 1] - x[:, 1]) + xs[:, 2] + xs[:, 3]
            err = float(np.linalg.norm(d) / np.linalg.norm(xs[:, 0]))
        out[name] = {"solves_per_s": world * 1e3 / ms, "ms_per_solve": ms,
                     "factor_ms": infos[-1].factor_ms, "refine_iterations": infos[-1].iterations,
                     "converged": bool(infos[-1].converged), "rel_err_vs_f512": err}
    out["chosen_over_plain"] = out["chosen"]["solves_per_s"] / out["plain"]["solves_per_s"]
    return out


def batched_section(hp, torch, dev, stream, sptr, args, world, dist):
    """4096 uneven overlap SPD systems (n in [16, 384]) in one graph-replayed
    persistent launch, plus batched Jacobi on the n <= 128 systems."""
    import numpy as np

    from quadprec_b200.workloads import batched_overlap_systems

    B = batched_overlap_systems(4096, seed=0)
    off = np.ascontiguousarray(B["offsets"], dtype=np.int64)
    count = len(off) - 1
    N = int(off[-1])
    ns = np.diff(off)
    dc = torch.from_numpy(np.ascontiguousarray(B["centers"])).to(dev)
    da = torch.from_numpy(B["alpha"]).to(dev)
    db = torch.from_numpy(np.stack([B["b"], np.zeros(N)], -1)).to(dev)
    dx = torch.empty((N, 2), dtype=torch.float64, device=dev)
    st = torch.zeros(count, dtype=torch.int32, device=dev)
    it = torch.zeros(count, dtype=torch.int32, device=dev)
    lib = hp.lib()

    def solve():
        hp.check(lib.hp_spd_solve_batched_dev(count, off.ctypes.data, dc.data_ptr(), da.data_ptr(), db.data_ptr(),
                                              dx.data_ptr(), st.data_ptr(), it.data_ptr(), 1e-28, 10, sptr))

    solve()  # captures the graph
    torch.cuda.synchronize()
    steps = max(2, args.spd_steps)
    if dist is not None:
        dist.barrier()
    s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(steps):
        solve()
    e0.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(s0.elapsed_time(e0) / steps, dist, dev)
    status = st.cpu().numpy()
    ok = int((status == 0).sum())
    acc = None
    fixp = os.path.join(REPO, "tests", "golden", "batched_4096_sample.npz")
    if os.path.exists(fixp):
        fx = np.load(fixp)
        xh = dx.cpu().numpy()
        errs = []
        for t, sidx in enumerate(fx["index"]):
            xg, xr = xh[off[sidx]:off[sidx + 1]], fx["x_star"][fx["x_offsets"][t]:fx["x_offsets"][t + 1]]
            d = (xg[:, 0] - xr[:, 0]) + (xg[:, 1] - xr[:, 1]) - xr[:, 2] - xr[:, 3]
            errs.append(float(np.linalg.norm(d) / np.linalg.norm(xr[:, 0])))
        acc = {"max_rel_err_vs_f512": max(errs), "systems_checked": len(errs),
               "n_range": [int(fx["n"].min()), int(fx["n"].max())],
               "kappa_range": [float(fx["kappa"].min()), float(fx["kappa"].max())],
               "sample": "48 systems spread over the sizes + the 16 largest cond_estimate (tests/golden/"
                         "batched_4096_sample.npz, mf_cholesky<8> solutions)"}
    out = {"workload": "4096 overlap SPD systems, n = 4*round(16*24^U/4) in [16, 384] (mean %.1f), random "
                       "3-D clusters (spacing 1.2-2.0 bohr), 4 exponents log-uniform in [0.01, 10], b ~ N(0,1); "
                       "each assembled in f128, factored and refined to max|dx| <= 1e-28 max|x|" % ns.mean(),
           "systems": count, "converged": ok, "ms_per_batch": ms,
           "systems_per_s": world * ok * 1e3 / ms,
           "f128_gflops_factor": world * float((ns.astype(np.float64) ** 3).sum() / 3.0) / (ms * 1e-3) / 1e9,
           "refine_iterations_max": int(it.cpu().numpy().max()),
           "accuracy": acc,
           "launch": "one persistent kernel (work queue, largest-first) replayed from a CUDA graph",
           "launch_shape": dict(zip(("threads_per_cta", "ctas_per_sm"), hp.batched_config()),
                                picked_by="autotuner (every candidate timed on this batch at the first call)")}
    # FP64-pipe roofline of the persistent kernel: the factorisations alone
    # are sum n^3/6 f128 multiply-adds of 29 FP64 instructions each
    # (reference-order Add + Mul); assembly, solves and refinement add more
    fp64_peak = getattr(args, "fp64_tflops", None)
    instr = float((ns.astype(np.float64) ** 3).sum() / 6.0) * 29.0
    achieved = world * instr / (ms * 1e-3) / 1e12  # T FP64 instructions / s
    out["roofline"] = {"bound": "fp64", "kernel": "batched_spd_kernel (persistent, graph-replayed)",
                       "achieved": achieved, "unit": "T FP64 instr/s (factorisation only)",
                       "peak": fp64_peak / 2.0 if fp64_peak else None,
                       "frac": achieved / (fp64_peak / 2.0) if fp64_peak else None,
                       "peak_source": "hp_measure_peaks DFMA loop, this run (TFLOP/s / 2)",
                       "algorithmic": "sum_s n_s^3/6 f128 multiply-adds x 29 FP64 instructions"}
    if getattr(args, "cpu_leg", False):
        out["cpu_baseline"] = cpu_batched_sample(B)
    # batched Jacobi on the n <= 128 systems
    sel = np.nonzero(ns <= 128)[0]
    joff = np.zeros(len(sel) + 1, dtype=np.int64)
    joff[1:] = np.cumsum(ns[sel])
    cen_sel = np.concatenate([B["centers"][off[i]:off[i + 1]] for i in sel])
    al_sel = np.concatenate([B["alpha"][off[i]:off[i + 1]] for i in sel])
    jc = torch.from_numpy(np.ascontiguousarray(cen_sel)).to(dev)
    ja = torch.from_numpy(al_sel).to(dev)
    mats = int((ns[sel] ** 2).sum())
    S = torch.empty(mats * 2, dtype=torch.float64, device=dev)
    hp.check(lib.hp_overlap_norm_dd_batched_dev(len(sel), joff.ctypes.data, jc.data_ptr(), ja.data_ptr(),
                                                S.data_ptr(), sptr))
    ev = torch.empty(int(joff[-1]) * 2, dtype=torch.float64, device=dev)
    vec = torch.empty_like(S)
    sw = torch.zeros(len(sel), dtype=torch.int32, device=dev)
    jst = torch.zeros(len(sel), dtype=torch.int32, device=dev)
    S_host = S.cpu().numpy() if getattr(args, "cpu_leg", False) else None  # the matrices, before the solver runs
    torch.cuda.synchronize()
    s1, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s1.record(stream)
    hp.check(lib.hp_f128_jacobi_eigen_batched_dev(len(sel), joff.ctypes.data, S.data_ptr(), 200, ev.data_ptr(),
                                                  vec.data_ptr(), sw.data_ptr(), jst.data_ptr(), sptr))
    e1.record(stream)
    torch.cuda.synchronize()
    jms = max_over_ranks(s1.elapsed_time(e1), dist, dev)
    sweeps = sw.cpu().numpy().astype(np.float64)
    nsel = ns[sel].astype(np.float64)
    rot = float((sweeps * nsel * (nsel - 1) / 2).sum())
    out["jacobi"] = {"matrices": int(len(sel)), "converged": int((jst.cpu().numpy() == 0).sum()), "ms": jms,
                     "matrices_per_s": world * len(sel) * 1e3 / jms, "rotations_per_s": world * rot / (jms * 1e-3),
                     "mean_sweeps": float(sweeps.mean())}
    if getattr(args, "cpu_leg", False):
        out["jacobi"]["cpu_baseline"] = cpu_jacobi_sample(S_host, ns[sel], ev.cpu().numpy())
    return out


def cpu_jacobi_sample(Sh, ns, evh, stride: int = 64) -> dict:
    """The reference's jacobi_eigen (crates/quad/src/linalg.rs:299-362,
    restated in the oracle) on a bounded sample of the batched Jacobi's
    matrices: every stride-th in size order, on 1 core and on all cores (one
    matrix per thread), each rate scaled to the whole set by sum n^3. Also the
    largest eigenvalue difference between the GPU's and the oracle's on the
    sample (both sorted; the rotation orders differ)."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    import oracle

    ns = ns.astype(np.int64)
    soff = np.concatenate([[0], np.cumsum(ns * ns)])
    eoff = np.concatenate([[0], np.cumsum(ns)])
    pick = np.argsort(ns, kind="stable")[::stride]

    def one(t):
        n = int(ns[t])
        return oracle.jacobi_eigen(Sh[2 * soff[t]:2 * soff[t + 1]].reshape(n, n, 2), n, 200)

    rates, res = {}, None
    cores = oracle.num_threads()
    for threads in (1, cores):
        t0 = time.perf_counter()
        if threads == 1:
            res = [one(t) for t in pick]
        else:
            with ThreadPoolExecutor(max_workers=threads) as ex:
                res = list(ex.map(one, pick))
        rates[threads] = len(pick) / (time.perf_counter() - t0)
    work = float((ns.astype(np.float64) ** 3).sum() / (ns[pick].astype(np.float64) ** 3).sum())
    diff = 0.0
    for t, (ev_c, _, _) in zip(pick, res):
        g = evh[2 * eoff[t]:2 * eoff[t + 1]].reshape(-1, 2)
        g = g[np.argsort(g[:, 0] + g[:, 1])]
        c = ev_c[np.argsort(ev_c[:, 0] + ev_c[:, 1])]
        d = np.abs((g[:, 0] - c[:, 0]) + (g[:, 1] - c[:, 1]))
        diff = max(diff, float(d.max() / np.abs(c[:, 0]).max()))
    whole = len(ns) / (len(pick) * work)  # sample rate -> matrices/s of the whole set
    return {"value": rates[cores] * whole, "unit": "matrices/s", "cores": cores,
            "kind": "port", "value_1_core": rates[1] * whole,
            "max_eigenvalue_diff_over_max_vs_gpu": diff,
            "sample": f"{len(pick)} of {len(ns)} matrices (every {stride}th in size order, n {int(ns[pick].min())}-"
                      f"{int(ns[pick].max())}), the reference's cyclic jacobi_eigen, rate scaled to the set by "
                      "sum n^3"}


ADJ_LATTICE = (5, 5, 10)  # 250 centres x 4 exponents = 1000 basis functions


def cpu_batched_sample(B, target_s: float = 15.0) -> dict:
    """The batch on the host cores (oracle.batched_refined: each system
    assembled in f128, reference f128 cholesky + solve_cholesky, refinement
    with f256 residuals; OpenMP over systems) on a bounded sample: every
    stride-th system in size order, the rate scaled to the whole batch by
    sum n^3 (the factorisations' share of the work)."""
    import numpy as np

    import oracle

    off = B["offsets"]
    ns = np.diff(off)
    order = np.argsort(ns, kind="stable")
    stride = 16
    while True:
        sel = order[::stride]
        sub = {"offsets": np.concatenate([[0], np.cumsum(ns[sel])]).astype(np.int64),
               "centers": np.concatenate([B["centers"][off[i]:off[i + 1]] for i in sel]),
               "alpha": np.concatenate([B["alpha"][off[i]:off[i + 1]] for i in sel]),
               "b": np.concatenate([B["b"][off[i]:off[i + 1]] for i in sel])}
        t0 = time.perf_counter()
        _, it = oracle.batched_refined(sub)
        dt = time.perf_counter() - t0
        if dt * 4 > target_s or stride <= 2:
            break
        stride //= 2
    w_all = float((ns.astype(np.float64) ** 3).sum())
    w_sub = float((ns[sel].astype(np.float64) ** 3).sum())
    est = dt * w_all / w_sub
    # one core on a sparser sample (every 8th system of the one above)
    sel1 = sel[::8]
    sub1 = {"offsets": np.concatenate([[0], np.cumsum(ns[sel1])]).astype(np.int64),
            "centers": np.concatenate([B["centers"][off[i]:off[i + 1]] for i in sel1]),
            "alpha": np.concatenate([B["alpha"][off[i]:off[i + 1]] for i in sel1]),
            "b": np.concatenate([B["b"][off[i]:off[i + 1]] for i in sel1])}
    prev = oracle.num_threads()
    oracle.set_threads(1)
    t0 = time.perf_counter()
    oracle.batched_refined(sub1)
    dt1 = time.perf_counter() - t0
    oracle.set_threads(prev)
    est1 = dt1 * w_all / float((ns[sel1].astype(np.float64) ** 3).sum())
    return {"value": len(ns) / est, "unit": "systems/s", "cores": oracle.num_threads(), "kind": "port",
            "value_1_core": len(ns) / est1,
            "sample": f"{len(sel)} of {len(ns)} systems (every {stride}th in size order, n {int(ns[sel].min())}-"
                      f"{int(ns[sel].max())}), {dt:.2f} s, scaled to the batch by sum n^3; all steps converged: "
                      f"{bool((it > 0).all())}; 1 core: {len(sel1)} systems (every {8 * stride}th), {dt1:.2f} s"}


def adjoint_fd_error(gR, ga):
    """Largest |g - g_fd| over the 56 parameters of tests/golden/adjoint_fd_1000.npz
    (f256 central differences, h = 1e-20), relative to the largest component."""
    import numpy as np

    p = os.path.join(REPO, "tests", "golden", "adjoint_fd_1000.npz")
    if not os.path.exists(p):
        return None
    fx = np.load(p)
    gmax = max(np.abs(gR[..., 0]).max(), np.abs(ga[..., 0]).max())
    errs = []
    for ci, c in enumerate(fx["centres"]):
        for comp in range(3):
            fd, g = fx["gR"][ci, comp], gR[c, comp]
            errs.append(abs(((g[0] - fd[0]) + (g[1] - fd[1])) - fd[2] - fd[3]))
    for qi, u in enumerate(fx["funcs"]):
        fd, g = fx["ga"][qi], ga[u]
        errs.append(abs(((g[0] - fd[0]) + (g[1] - fd[1])) - fd[2] - fd[3]))
    return {"max_abs_err_over_max_component": float(max(errs) / gmax), "parameters": len(errs),
            "reference": "f256 central differences, h = 1e-20 (tests/golden/adjoint_fd_1000.npz)"}


def adjoint_section(hp, torch, dev, stream, sptr, args, world, dist):
    """Gradient of L = b^T S^-1 b wrt 750 centre coordinates and 1000
    log-exponents (n = 1000): assembly + refined solve + adjoint sweep."""
    import ctypes

    import numpy as np

    from quadprec_b200.workloads import overlap_spd_problem

    cen, alpha, b = overlap_spd_problem(*ADJ_LATTICE, seed=0)
    n = len(alpha)
    nc = n // 4
    co = np.arange(n, dtype=np.int32) // 4
    dcen = torch.from_numpy(np.ascontiguousarray(cen)).to(dev)
    dal = torch.from_numpy(alpha).to(dev)
    db = torch.from_numpy(np.stack([b, np.zeros(n)], -1)).to(dev)
    dco = torch.from_numpy(co).to(dev)
    loss = torch.empty(2, dtype=torch.float64, device=dev)
    gR = torch.empty((nc, 3, 2), dtype=torch.float64, device=dev)
    ga = torch.empty((n, 2), dtype=torch.float64, device=dev)
    lib = hp.lib()
    out = {"workload": f"dL/dtheta for L = b^T S^-1 b, n = {n} s-Gaussians (250 jittered 5x5x10 lattice centres x 4 "
                       "exponents), theta = 750 centre coordinates + 1000 log-exponents", "unit": "gradients/s"}
    grads = {}
    for name, mode in (("chosen", hp.OZAKI), ("plain", hp.PLAIN)):
        info = hp.RefineInfo()

        def one():
            hp.check(lib.hp_overlap_adjoint_dev(n, dcen.data_ptr(), dal.data_ptr(), db.data_ptr(), dco.data_ptr(), nc,
                                                mode, loss.data_ptr(), gR.data_ptr(), ga.data_ptr(),
                                                ctypes.byref(info), sptr))

        one()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        steps = max(2, args.spd_steps)
        s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(steps):
            one()
        e0.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(s0.elapsed_time(e0) / steps, dist, dev)
        grads[name] = (gR.cpu().numpy().copy(), ga.cpu().numpy().copy())
        out[name] = {"gradients_per_s": world * 1e3 / ms, "ms_per_gradient": ms, "converged": bool(info.converged),
                     "accuracy_vs_f256_fd": adjoint_fd_error(*grads[name])}
    out["chosen_over_plain"] = out["chosen"]["gradients_per_s"] / out["plain"]["gradients_per_s"]
    if getattr(args, "cpu_leg", False):
        import oracle

        t0 = time.perf_counter()
        _, cgR, cga = oracle.adjoint_f128_refined(cen, alpha, b, co, nc)
        dt = time.perf_counter() - t0
        prev = oracle.num_threads()
        oracle.set_threads(1)
        t0 = time.perf_counter()
        oracle.adjoint_f128_refined(cen, alpha, b, co, nc)
        dt1 = time.perf_counter() - t0
        oracle.set_threads(prev)
        # every component of both GPU gradients against the oracle's full f128 gradient
        ref = np.concatenate([np.asarray(cgR).reshape(-1, 2)[:, 0], np.asarray(cga).reshape(-1, 2)[:, 0]])
        scale = float(np.max(np.abs(ref)))
        for name, (gR_, ga_) in grads.items():
            got = np.concatenate([gR_.reshape(-1, 2), ga_.reshape(-1, 2)])
            want = np.concatenate([np.asarray(cgR).reshape(-1, 2), np.asarray(cga).reshape(-1, 2)])
            err = np.abs((got[:, 0] - want[:, 0]) + (got[:, 1] - want[:, 1]))
            out[name]["accuracy_vs_oracle_gradient"] = {
                "max_abs_err_over_max_component": float(err.max() / scale), "components": int(len(err)),
                "reference": "the oracle's full gradient (reference f128 cholesky + solve_cholesky, f256 residuals, "
                             "f128 contraction)"}
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "gradients/s", "cores": oracle.num_threads(),
                               "kind": "port", "value_1_core": 1.0 / dt1,
                               "accuracy_vs_f256_fd": adjoint_fd_error(cgR, cga),
                               "sample": f"one full gradient, {dt:.2f} s ({dt1:.2f} s on 1 core): S in f128, lambda "
                                         "from the reference's "
                                         "f128 cholesky + solve_cholesky refined with f256 residuals, then the "
                                         "f128 contraction -lambda^T dS lambda (OpenMP rows)"}
    return out


CH_N = 512  # the plain f128 Cholesky solve of the reference's README matrix


def cholesky512_section(hp, torch, dev, stream, sptr, args, world, dist):
    """The reference's own plain path at n = 512: cholesky + solve_cholesky
    (crates/quad/src/linalg.rs:42-126) of A_ij = 1/(i+j+1) + I, b = ones, no
    refinement. One step = one factorisation + both triangular solves of a
    fresh copy of A (device-resident; hp_f128_cholesky_dev synchronises its
    stream to report a failed pivot, as the reference returns its Result)."""
    import ctypes

    import numpy as np

    from quadprec_b200.workloads import shifted_hilbert

    n = CH_N
    a, b = shifted_hilbert(n)
    lib = hp.lib()
    dA = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    dL = torch.empty_like(dA)
    dx = torch.empty_like(db)
    pv, val = ctypes.c_int64(-1), ctypes.c_double(0.0)

    def one():
        dL.copy_(dA)
        dx.copy_(db)
        hp.check(lib.hp_f128_cholesky_dev(dL.data_ptr(), n, ctypes.byref(pv), ctypes.byref(val), sptr))
        hp.check(lib.hp_f128_solve_cholesky_dev(dL.data_ptr(), dx.data_ptr(), n, sptr))

    for _ in range(3):
        one()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    steps = 20
    s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(steps):
        one()
    e0.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(s0.elapsed_time(e0) / steps, dist, dev)
    x_dev = dx.cpu().numpy()
    # end to end: the host-pointer entry points, as a caller of the Rust API would
    L = np.empty_like(a)
    x = np.empty_like(b)
    ha = np.ascontiguousarray(a)

    def one_host():
        np.copyto(L, ha)
        hp.check(lib.hp_f128_cholesky(L.ctypes.data, n, ctypes.byref(pv), ctypes.byref(val)))
        hp.check(lib.hp_f128_solve_cholesky(L.ctypes.data, b.ctypes.data, x.ctypes.data, n))

    one_host()
    t0 = time.perf_counter()
    for _ in range(steps):
        one_host()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / steps, dist, dev)
    fma = n ** 3 / 6.0 + n * n  # f128 multiply-adds: factorisation + two triangular solves
    fp64_peak = getattr(args, "fp64_tflops", None)
    instr_rate = 29.0 * fma / (ms * 1e-3) / 1e12
    out = {"workload": "plain f128 Cholesky solve (cholesky + solve_cholesky), n = 512, A_ij = 1/(i+j+1) + I "
                       "(README matrix), b = ones, no refinement", "n": n, "unit": "solves/s",
           "solves_per_s": world * 1e3 / ms, "ms_per_solve": ms,
           "e2e": {"solves_per_s": world * 1e3 / e2e_ms, "ms_per_solve": e2e_ms,
                   "path": "hp_f128_cholesky + hp_f128_solve_cholesky (host pointers, copies inside)",
                   "h2d_bytes_per_step": int(n * n * 16 * 2 + n * 16), "d2h_bytes_per_step": int(n * n * 16 + n * 16)},
           "roofline": {"bound": "fp64", "achieved": instr_rate, "unit": "T FP64 instr/s",
                        "peak": fp64_peak / 2.0 if fp64_peak else None,
                        "frac": instr_rate / (fp64_peak / 2.0) if fp64_peak else None,
                        "algorithmic": "(n^3/6 + n^2) f128 multiply-adds x 29 FP64 instructions (reference Add + Mul)",
                        "peak_source": "hp_measure_peaks DFMA loop, this run (TFLOP/s / 2)"},
           "f128_gflops": world * 2.0 * fma / (ms * 1e-3) / 1e9}
    if getattr(args, "cpu_leg", False):
        import oracle

        res = {}
        for cores in (oracle.num_threads(), 1):
            prev = oracle.num_threads()
            oracle.set_threads(cores)
            t0 = time.perf_counter()
            Lc = oracle.cholesky(a, n)
            xc = oracle.solve_cholesky(Lc, b, n)
            res[cores] = time.perf_counter() - t0
            oracle.set_threads(prev)
        d = (x_dev[:, 0] - xc[:, 0]) + (x_dev[:, 1] - xc[:, 1])
        out["cpu_baseline"] = {"value": 1.0 / res[max(res)], "unit": "solves/s", "cores": max(res), "kind": "port",
                               "value_1_core": 1.0 / res[1],
                               "gpu_vs_cpu_normwise_diff": float(np.linalg.norm(d) / np.linalg.norm(xc[:, 0])),
                               "sample": f"one full solve on all cores ({res[max(res)]:.3f} s) and on 1 core "
                                         f"({res[1]:.3f} s): the reference's cholesky + solve_cholesky restated"}
    return out


def cpu_spd_sample() -> dict:
    """The same computation on the host cores: the reference's f128 cholesky +
    solve_cholesky refined with f256 residuals to the same 1e-28 stopping rule
    (oracle.spd_solve_refined; the reference's own solve_spd_f128 refines
    with f128 residuals and stalls near 1e-17 on this matrix), plus the
    assembly of S."""
    import numpy as np

    import oracle
    from quadprec_b200.workloads import overlap_spd_problem

    cen, alpha, b = overlap_spd_problem(*SPD_LATTICE, seed=0)
    n = len(alpha)
    times = {}
    prev = oracle.num_threads()
    for cores in (prev, 1):
        oracle.set_threads(cores)
        t0 = time.perf_counter()
        S = oracle.overlap_norm_dd(cen, alpha)
        x, steps = oracle.spd_solve_refined(S, b, n)
        times[cores] = time.perf_counter() - t0
    oracle.set_threads(prev)
    dt = times[prev]
    fix = os.path.join(REPO, "tests", "golden", "overlap_5x10x10.npz")
    err = None
    if os.path.exists(fix):
        xs = np.load(fix)["x_star"]
        d = (xs[:, 0] - x[:, 0]) + (xs[:, 1] - x[:, 1]) + xs[:, 2] + xs[:, 3]
        err = float(np.linalg.norm(d) / np.linalg.norm(xs[:, 0]))
    return {"value": 1.0 / dt, "unit": "solves/s", "cores": oracle.num_threads(), "kind": "port",
            "value_1_core": 1.0 / times[1], "rel_err_vs_f512": err,
            "sample": f"one full solve of the same n={n} system, {dt:.2f} s ({times[1]:.2f} s on 1 core): assembly "
                      "of S in f128, the reference's f128 cholesky + solve_cholesky (crates/quad/src/linalg.rs:42-126) "
                      f"and {steps} refinement steps with f256 residuals (mf_gemv semantics, "
                      "multifloat/linalg.rs:17-37), OpenMP rows"}


def profile_case_spd(args):
    """One overlap SPD solve per mode (chosen, then plain): the command ncu captures."""
    import torch

    import quadprec_b200 as hp

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    args.spd_steps = max(1, args.steps)
    out = spd_section(hp, torch, dev, stream, stream.cuda_stream, args, 0, 1, None)
    print(json.dumps(out), file=sys.stderr)
    return 0


def profile_case_chol512(args):
    """Plain f128 Cholesky solves at n = 512 (config 1), warmup + steps of them:
    the command ncu captures."""
    import ctypes

    import torch

    import quadprec_b200 as hp
    from quadprec_b200.workloads import shifted_hilbert

    dev = torch.device("cuda", 0)
    sptr = torch.cuda.current_stream(dev).cuda_stream
    n = CH_N
    a, b = shifted_hilbert(n)
    lib = hp.lib()
    dA = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    dL = torch.empty_like(dA)
    dx = torch.empty_like(db)
    pv, val = ctypes.c_int64(-1), ctypes.c_double(0.0)
    for _ in range(args.warmup + args.steps):
        dL.copy_(dA)
        dx.copy_(db)
        hp.check(lib.hp_f128_cholesky_dev(dL.data_ptr(), n, ctypes.byref(pv), ctypes.byref(val), sptr))
        hp.check(lib.hp_f128_solve_cholesky_dev(dL.data_ptr(), dx.data_ptr(), n, sptr))
    torch.cuda.synchronize()
    print("profile case done", file=sys.stderr)
    return 0


def profile_case_f256(args):
    """Chosen-path f256 GEMMs at m = n = k = 1024 on the benchmark's operands
    (double-double entries widened to four limbs): the command ncu captures."""
    import torch

    import quadprec_b200 as hp
    from quadprec_b200.workloads import dd_to_qd, gemm_operands

    n4 = 1024
    a, b = gemm_operands(n4, n4, n4, seed=0)
    A = torch.from_numpy(dd_to_qd(a)).cuda()
    B = torch.from_numpy(dd_to_qd(b)).cuda()
    C = torch.empty((n4, n4, 4), dtype=torch.float64, device="cuda")
    sptr = torch.cuda.current_stream().cuda_stream
    for _ in range(args.warmup + args.steps):
        hp.f256_gemm_dev(A, B, C, n4, n4, n4, hp.OZAKI, stream=sptr)
    torch.cuda.synchronize()
    print("profile case done", file=sys.stderr)
    return 0


def profile_case_e2e(args):
    """The host-pointer f128 GEMM at 2048^3 from pinned host buffers, with the
    library's timeline marks on: per call, the device times (ms from the
    call's start) at which B's first panel and all operands have landed, the
    first C block is back, the last block is computed and all of C is back."""
    import ctypes

    import torch

    import quadprec_b200 as hp
    from quadprec_b200.workloads import gemm_operands

    a_np, b_np = gemm_operands(M, N, K, seed=0)
    ha, hb = torch.from_numpy(a_np).pin_memory(), torch.from_numpy(b_np).pin_memory()
    hc = torch.empty((M, N, 2), dtype=torch.float64).pin_memory()
    lib = hp.lib()
    for _ in range(args.warmup):
        hp.check(lib.hp_f128_gemm(ha.data_ptr(), hb.data_ptr(), hc.data_ptr(), M, N, K, hp.OZAKI))
    for _ in range(args.steps):
        lib.hp_profile_enable(1)
        t0 = time.perf_counter()
        hp.check(lib.hp_f128_gemm(ha.data_ptr(), hb.data_ptr(), hc.data_ptr(), M, N, K, hp.OZAKI))
        wall = (time.perf_counter() - t0) * 1e3
        ms = (ctypes.c_double * 32)()
        names = ctypes.create_string_buffer(1024)
        cnt = lib.hp_profile_read(ms, 32, names, 1024)
        lib.hp_profile_enable(0)
        t, marks = 0.0, []
        for nm, d in zip(names.value.decode().split(","), ms[:cnt]):
            t += d
            marks.append(f"{nm}={t:.3f}")
        print(f"call {wall:.3f} ms (host clock): " + " ".join(marks), flush=True)
    return 0


# ---------------------------------------------------------------- main arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-spd", action="store_true", help="skip the overlap SPD solve section")
    ap.add_argument("--spd-steps", type=int, default=3)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched SPD / Jacobi section")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint section")
    ap.add_argument("--profile-case", nargs="?", const="gemm", default=None, choices=["gemm", "spd", "batched", "chol512", "f256", "e2e"],
                    help="only run warmup + steps of one chosen-path workload (for ncu captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_case == "gemm":
        return profile_case(args)
    if args.profile_case == "spd":
        return profile_case_spd(args)
    if args.profile_case == "chol512":
        return profile_case_chol512(args)
    if args.profile_case == "f256":
        return profile_case_f256(args)
    if args.profile_case == "e2e":
        return profile_case_e2e(args)
    if args.profile_case == "batched":
        import torch

        import quadprec_b200 as hp

        dev = torch.device("cuda", 0)
        stream = torch.cuda.current_stream(dev)
        out = batched_section(hp, torch, dev, stream, stream.cuda_stream, args, 1, None)
        print(json.dumps(out), file=sys.stderr)
        return 0

    import numpy as np
    import torch

    world, rank, local, dist = init_dist("nccl")
    torch.cuda.set_device(local)

    import quadprec_b200 as hp
    from quadprec_b200.workloads import gemm_operands

    assert hp.device_ok(), "no sm_100 device"
    a_np, b_np = gemm_operands(M, N, K, seed=rank)
    dev = torch.device("cuda", local)
    A = torch.from_numpy(a_np).to(dev)
    B = torch.from_numpy(b_np).to(dev)
    C = torch.empty((M, N, 2), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(mode, steps, warmup):
        for _ in range(warmup):
            hp.f128_gemm_dev(A, B, C, M, N, K, mode, stream=sptr)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        evs = []
        for _ in range(steps):
            flush.fill_(1.0)  # L2 flush, outside the timed interval
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            hp.f128_gemm_dev(A, B, C, M, N, K, mode, stream=sptr)
            e.record(stream)
            evs.append((s, e))
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(sum(s.elapsed_time(e) for s, e in evs) / steps, dist, dev)

    # roofline denominators measured on this device (DFMA loop, tcgen05 kind::i8 loop)
    pk = hp.measure_peaks(5)
    args.fp64_tflops = pk["fp64_tflops"]
    args.cpu_leg = rank == 0 and world == 1 and not args.no_cpu

    flops = 2.0 * M * N * K
    clk = ClockSampler(local)
    clk.start()
    ms_chosen = timed(hp.OZAKI, args.steps, args.warmup)
    clocks = clk.stop()
    ms_plain = timed(hp.PLAIN, args.plain_steps, 1)

    # correctness spot check of the timed output against the plain result
    hp.f128_gemm_dev(A, B, C, M, N, K, hp.OZAKI, stream=sptr)
    torch.cuda.synchronize()
    c_oz = C.cpu().numpy()
    hp.f128_gemm_dev(A, B, C, M, N, K, hp.PLAIN, stream=sptr)
    torch.cuda.synchronize()
    c_pl = C.cpu().numpy()
    diff = (c_oz[..., 0] - c_pl[..., 0]) + (c_oz[..., 1] - c_pl[..., 1])
    absab = np.abs(a_np[..., 0]) @ np.abs(b_np[..., 0])
    rel_err = float(np.linalg.norm(diff) / np.linalg.norm(absab))
    # errors against the f512 oracle (fixture of the seed-0 operands)
    err_f512 = ({"chosen": f512_errors(c_oz, a_np, b_np, "f128_gemm_2048"),
                 "plain": f512_errors(c_pl, a_np, b_np, "f128_gemm_2048"),
                 "bound": 4 * K * 2.0 ** -104} if rank == 0 else None)

    # phase timing of one chosen-path step (dominant kernel roofline)
    flush.fill_(1.0)
    torch.cuda.synchronize()
    hp.profile_enable(True)
    hp.f128_gemm_dev(A, B, C, M, N, K, hp.OZAKI, stream=sptr)
    phases = hp.profile_read()
    hp.profile_enable(False)

    L = 30
    hbm_gbs, bf16_tf, peak_kind = peaks()
    i8_peak = pk["i8_tops"]
    mm = phases.get("i8_gemm", float("nan"))
    i8_tops = L * 2.0 * M * N * K / (mm * 1e-3) / 1e12
    res_ms = phases.get("residues", float("nan"))
    res_bytes = 2 * (M * K * 16) + L * (M * K + N * K)
    crt_ms = phases.get("crt", float("nan"))
    crt_bytes = L * M * N + M * N * 16
    roofline = {"bound": "tensor", "kernel": "i8_gemm_pair_kernel (tcgen05.mma.cta_group::2 kind::i8 on CTA "
                "pairs, M = 256, one launch for all 30 moduli)", "achieved": i8_tops, "peak": i8_peak, "unit": "TOPS (int8)",
                "frac": i8_tops / i8_peak, "traffic": I8_GEMM_TRAFFIC_BYTES,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch at 2048^3",
                "peak_source": ("measured in this run by hp_measure_peaks: tcgen05.mma kind::i8 (u8, M=128, "
                                "N=256, K=32) back to back on every SM, CUDA events; for comparison 2 x the "
                                f"{peak_kind} dense bf16 figure = {2.0 * bf16_tf:.1f} TOPS"),
                "frac_of_2x_bf16": i8_tops / (2.0 * bf16_tf),
                "algorithmic": f"{L} moduli x 2mnk int8 ops = {L * 2.0 * M * N * K:.3e} per launch"}
    phase_report = {k: round(v, 4) for k, v in phases.items()}
    phase_roofline = {
        "residues_hbm_frac": (res_bytes / (res_ms * 1e-3) / 1e9) / hbm_gbs if res_ms == res_ms else None,
        "crt_hbm_frac": (crt_bytes / (crt_ms * 1e-3) / 1e9) / hbm_gbs if crt_ms == crt_ms else None,
    }

    # end to end through the host-pointer C ABI (pinned host buffers)
    ha = torch.from_numpy(a_np).pin_memory()
    hb = torch.from_numpy(b_np).pin_memory()
    hc = torch.empty((M, N, 2), dtype=torch.float64).pin_memory()
    lib = hp.lib()
    for _ in range(2):
        hp.check(lib.hp_f128_gemm(ha.data_ptr(), hb.data_ptr(), hc.data_ptr(), M, N, K, hp.OZAKI))
    barrier()
    e2e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        hp.check(lib.hp_f128_gemm(ha.data_ptr(), hb.data_ptr(), hc.data_ptr(), M, N, K, hp.OZAKI))
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, dist, dev)

    more = gemm_more_section(hp, torch, dev, stream, sptr, world, dist)
    chol512 = cholesky512_section(hp, torch, dev, stream, sptr, args, world, dist)
    spd = None if args.no_spd else spd_section(hp, torch, dev, stream, sptr, args, rank, world, dist)
    batched = None if args.no_batched else batched_section(hp, torch, dev, stream, sptr, args, world, dist)
    adjoint = None if args.no_adjoint else adjoint_section(hp, torch, dev, stream, sptr, args, world, dist)

    cpu = None
    if args.cpu_leg:
        cpu = cpu_sample_gflops()
        cpu["value_1_core"] = cpu_sample_gflops(target_s=4.0, threads=1)["value"]
        if spd is not None:
            spd["cpu_baseline"] = cpu_spd_sample()

    value = world * flops / (ms_chosen * 1e-3) / 1e9
    plain_value = world * flops / (ms_plain * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_chosen, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8 residues -> int32 (exact) + f64 EFT (double-double result)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "m": M, "n": N, "k": K, "mode": "ozaki (Ozaki-II, 30 int8 moduli)",
                   "l2": "flushed between timed steps (256 MiB write, untimed)",
                   "parallelism": f"{world} independent GEMMs (one per GPU)"},
        "plain": {"value": plain_value, "unit": "GFLOP/s", "ms_per_step": ms_plain, "steps": args.plain_steps,
                  "mode": "plain CUDA-core dd FMA, bit-identical to the reference"},
        "chosen_over_plain": value / plain_value,
        "normwise_rel_err_vs_plain": rel_err,
        "err_vs_f512": err_f512,
        "peaks_measured": {"fp64_tflops": pk["fp64_tflops"], "i8_tops": pk["i8_tops"],
                           "how": "hp_measure_peaks: DFMA loop (8 chains per thread, 8 CTAs of 256 per SM) and "
                                  "tcgen05.mma kind::i8 loop (one CTA per SM), best of 5, CUDA events"},
        "e2e": {"value": world * flops / e2e_s / 1e9, "unit": "GFLOP/s",
                "h2d_bytes_per_step": int(2 * M * K * 16), "d2h_bytes_per_step": int(M * N * 16),
                "path": "hp_f128_gemm (host pointers, pinned), copies inside the timed region"},
        "roofline": roofline, "phases_ms": phase_report, "phase_roofline": phase_roofline,
        "gpu_launches": 4 * args.steps,  # exponents, residues, tcgen05 GEMM, CRT per step
        "clocks": clocks,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    line["gemm_more"] = more
    line["cholesky_512"] = chol512
    if spd is not None:
        line["spd"] = spd
    if batched is not None:
        line["batched"] = batched
    if adjoint is not None:
        line["adjoint"] = adjoint
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
