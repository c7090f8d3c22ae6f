"""Benchmark of the SHORE L1 volume fit (voxels/s).

Workload: the brain-sized synthetic volume (96 x 114 x 96 grid, ellipsoidal
mask of 299,432 voxels, CS-DSI table with N = 259, radial order 6 -> K = 72,
zeta 700), L1 FISTA with a fixed alpha = 0.01 at the reference defaults
(max_iter 1000, tol 1e-6).  One step = one whole-volume fit.  Both GPU paths
run on the same volume: FP64 (the reference arithmetic, FISTA on FP64 DMMA
tensor cores) and mixed (int8 digit-slice Gram products on tcgen05 tensor
cores, FP64 state); `value` is the faster of the two, both being within the
1e-5 coefficient tolerance of FP64 (the line states which, and the measured
error of the mixed path against the FP64 path).

* value   voxels/s with the volume already resident in HBM (device entry
          point), CUDA events on the fit stream, max over ranks.
* e2e     the same fit through the reference-facing C ABI with host buffers
          in page-locked memory, every step: the library reads the masked rows
          of the host volume over the bus, fits, and copies the coefficient
          volume back (host clock around the blocking call).
* roofline  the dominant kernel (FP64 FISTA on DMMA tensor cores): algorithmic
          FLOPs = executed voxel-iterations x (2K^2 + 8K) per launch (the dense
          Gram form) over the kernel's event-timed duration, against the FP64
          DMMA peak measured live by libcsdpeak (no FP64 figure exists in
          MEASURED_PEAKS.json).  The kernel skips k-steps whose iterate entries
          are all exactly zero, so the tensor FLOPs it executes (counted on the
          device, also reported) are fewer than the algorithmic count.
* fwd_bwd the metric's second half: the differentiable fit of 50,000 voxels
          (fit + RTOP + 362-direction ODF, then backward to the signals and the
          hyper-parameter), voxels/s for L1 and Tikhonov, and the ratio of the
          forward+backward step to the forward step.
* graddev the per-voxel-design fit (radial order 8, a gradient-deviation
          tensor and 0-15 % dropped samples per voxel) on 300k voxels.
* pipeline the hypergradient alpha selection pipeline (8 steps on a held-out
          10 % of the samples, final fit, peaks, RTOP / MSD) on the same
          volume, host clock, with the held-out error of the reference's own
          alpha selections beside it.
* cpu_baseline  the CPU FP64 oracle (a restatement of the reference's rayon
          path: the Rust reference cannot be built without cargo) on all host
          threads, on a bounded sample of the same voxels.

``--impl reference`` times that CPU path alone, as the reference arm.
Multi-GPU: `--gpus N` runs N ranks (under torchrun, or launched by this
script itself when no launcher set WORLD_SIZE).  The line's `value` is weak
scaling: every rank fits its own copy of the volume (independent subjects; no
collective in the data path).  The `sharded` block is strong scaling: one
volume split across the ranks, and the row gather that reassembles it.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import socket
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SHORE L1-fit voxels/s, mixed vs FP64 GPU at \u22641e-5 rel err; fwd+bwd voxels/s"
FWD_BWD_GRID = (50, 50, 20)  # the differentiable-fit workload: 50,000 voxels, radial order 6
GRADDEV_VOXELS = 300_000     # per-voxel-design workload (radial order 8): configuration 3's size
WORKLOAD = "brain300k"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--profile-case", choices=["graddev2k", "graddev2k-mixed", "diff50k", "peaks108k", "fista125k",
                                               "kkt64k", "icls64k", "tikhonov64k"],
                    help="run one small profiling workload instead of the benchmark")
    ap.add_argument("--workload", choices=["brain300k", "grid64k"], default="brain300k",
                    help="brain300k: the benchmark volume; grid64k: 40^3 fully masked (profiling case)")
    return ap.parse_args()


def fit_kwargs():
    return dict(alpha_mode="fixed", alpha=0.01, max_iter=1000, tol=1e-6, radial_order=6, zeta=700.0)


def load_phantom():
    from cs_dmri_b200.phantom import config_phantom
    return config_phantom(WORKLOAD)


def select_workload(name: str) -> None:
    global WORKLOAD
    WORKLOAD = name


# ------------------------------------------------------------------ CPU leg

def cpu_sample(ph, target_s: float, threads: int = 0):
    """A strided sample of the masked voxels (every k-th in x-y-z order, so it
    spans the whole mask) sized for about `target_s` seconds of the CPU FP64
    oracle on `threads` host threads (0 = all), from one untimed probe fit.
    Returns (sample voxel signals as a (V, 1, 1, N) volume, its mask,
    the stride, the thread count)."""
    from oracle import oracle as O

    ids = np.flatnonzero(ph.mask.ravel())
    n = ph.data.shape[-1]
    flat = ph.data.reshape(-1, n)
    cores = threads or O.cpu_count()

    def volume(stride):
        sub = np.ascontiguousarray(flat[ids[::stride]]).reshape(-1, 1, 1, n)
        return sub, np.ones(sub.shape[:3], bool)

    stride = max(1, len(ids) // max(256, 32 * cores))
    for _ in range(2):  # the second probe runs at about a quarter of the target length
        sub, m = volume(stride)
        t = cpu_fit(ph, sub, m, threads)
        rate = len(sub) / max(t, 1e-3)
        stride = max(1, int(len(ids) / max(rate * target_s * (0.25 if _ == 0 else 1.0), 1.0)))
    sub, m = volume(stride)
    return sub, m, stride, cores


def cpu_fit(ph, sub, m, threads: int) -> float:
    """Seconds of one oracle fit of the sample volume."""
    from oracle import oracle as O
    t = time.perf_counter()
    O.shore_fit(sub, ph.bvals, ph.bvecs, m, big_delta=ph.big_delta, small_delta=ph.small_delta,
                n_threads=threads, return_coef64=False, **fit_kwargs())
    return time.perf_counter() - t


def cpu_sample_rate(ph, target_s: float, threads: int = 0):
    """Voxels/s of the CPU FP64 oracle on a strided sample of the volume."""
    sub, m, stride, cores = cpu_sample(ph, target_s, threads)
    t = cpu_fit(ph, sub, m, threads)
    return len(sub) / t, len(sub), cores, t, stride


def bench_config(ph) -> dict:
    """The workload, identical in both arms."""
    X, Y, Z, N = ph.data.shape
    return {"workload": WORKLOAD, "voxels": ph.n_voxels, "grid": [X, Y, Z], "N": N, "K": 72, "alpha": 0.01,
            "solver": "L1 FISTA, fixed alpha 0.01, max_iter 1000, tol 1e-6 (reference stopping rule)",
            "l2": f"inputs larger than L2 ({ph.data.nbytes / 1e9:.2f} GB volume per step)"}


# ------------------------------------------------------------------ clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts only once the sampler is producing samples
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.02)
            self.start = len(self.lines)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[max(0, getattr(self, "start", 0) - 1):]  # from the last sample before the region
        for ln in lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, val in zip(names, p[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


# ------------------------------------------------------------------ helpers

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def traffic_from_profile(voxels: int, parked: float):
    """DRAM bytes of one fit's FISTA passes from the committed ncu summary of
    the two-pass schedule: a per-voxel figure plus one per parked voxel (its
    state written at the cap and read back), times this run's counts."""
    p = ROOT / "profiles" / "k_fista_v3_twopass_fista125k.md"
    if not p.exists():
        return None
    t = p.read_text()
    a = re.search(r"traffic_bytes_per_voxel:\s*([0-9.eE+]+)", t)
    b = re.search(r"traffic_bytes_per_parked_voxel:\s*([0-9.eE+]+)", t)
    return float(a.group(1)) * voxels + float(b.group(1)) * parked if a and b else None


def fp64_peak_tflops(device: int):
    import ctypes
    lib = ctypes.CDLL(str(ROOT / "cs_dmri_b200" / "libcsdpeak.so"))
    a, b = ctypes.c_double(), ctypes.c_double()
    vals = []
    for _ in range(3):
        if lib.csd_peak_fp64(device, ctypes.byref(a), ctypes.byref(b)) != 0:
            return None, None
        vals.append((a.value, b.value))
    return max(v[0] for v in vals), max(v[1] for v in vals)


# ------------------------------------------------------------------ arms

def run_reference(args):
    """The reference arm: the CPU FP64 oracle (the reference's per-voxel
    algorithm restated; the Rust reference needs cargo, absent here) on all
    host threads.  Every step fits the same strided sample of the masked
    voxels (every k-th voxel in mask order), sized for about two seconds; the
    line reports the measured time of one step and the sample's voxels/s."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    ph = load_phantom()
    from oracle import oracle as O
    O.build()
    sub, m, stride, cores = cpu_sample(ph, 2.0, threads=0)
    times = []
    for i in range(args.warmup + args.steps):
        t = cpu_fit(ph, sub, m, 0)
        if i >= args.warmup:
            times.append(t)
    sec = sum(times)
    value = len(sub) * args.steps / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded CS-DSI multi-tensor phantom, S0 1000, SNR 25)",
        "config": bench_config(ph),
        "voxels_per_step": len(sub),
        "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": cores, "kind": "port",
                         "sample": f"every masked voxel at stride {stride} ({len(sub)} of {ph.n_voxels}) per step, "
                                   "CPU FP64 oracle on all host threads; ms_per_step is that sample's fit"},
        "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup(args)
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    from cs_dmri_b200 import _abi, shore_fit, shore_fit_device

    ph = load_phantom()
    kw = fit_kwargs()
    X, Y, Z, N = ph.data.shape
    K = 72
    d_data = torch.from_numpy(ph.data).to(f"cuda:{device}")
    d_mask = torch.from_numpy(ph.mask).to(f"cuda:{device}")
    coeffs = torch.empty((X, Y, Z, K), dtype=torch.float32, device=f"cuda:{device}")
    stream = torch.cuda.Stream(device=device)

    def device_step(precision="fp64"):
        c, res = shore_fit_device(d_data, d_mask, ph.bvals, ph.bvecs, coefficients=coeffs, stream=stream,
                                  device=device, big_delta=ph.big_delta, small_delta=ph.small_delta,
                                  precision=precision, **kw)
        return res

    # ---- value: inputs resident in HBM (1.09 GB volume > 126 MB L2 per step)
    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize(device)
    barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kernel_ms, tensor_flops, launches, iters, parked, warps = [], [], 0, [], [], set()
    with ClockSampler(device) as clocks:
        torch.cuda.synchronize(device)
        ev0.record(stream)
        for _ in range(args.steps):
            res = device_step()
            tm = _abi.last_timing(device)
            kernel_ms.append(tm.ms_solve_kernel)
            tensor_flops.append(tm.tensor_flops)
            parked.append(tm.fista_parked)
            warps.add(tm.fista_warps)
            iters.append(res.total_iterations)
            launches += tm.launches
        ev1.record(stream)
        torch.cuda.synchronize(device)
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, world, torch.device("cuda", device))
    V = int(ph.mask.sum())
    value = world * V * args.steps / (ms / 1e3)

    # ---- the mixed-precision path on the same volume
    for _ in range(args.warmup):
        device_step("mixed")
    torch.cuda.synchronize(device)
    barrier(world)
    mix_kernel_ms, mix_ops, mix_rerun, mix_launches = [], [], [], 0
    with ClockSampler(device) as mix_clocks:
        torch.cuda.synchronize(device)
        ev0.record(stream)
        for _ in range(args.steps):
            device_step("mixed")
            tm = _abi.last_timing(device)
            mix_kernel_ms.append(tm.ms_mixed_kernel)
            mix_ops.append(tm.int8_tensor_ops)
            mix_rerun.append(int(tm.fp64_rerun_voxels))
            mix_launches += tm.launches
        ev1.record(stream)
        torch.cuda.synchronize(device)
    ms_mix = max_over_ranks(ev0.elapsed_time(ev1), world, torch.device("cuda", device))
    value_mix = world * V * args.steps / (ms_mix / 1e3)
    # coefficient error of the mixed path against the FP64 path (FP64 outputs)
    import numpy as np
    common = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, device=device, return_coef64=True,
                  diagnostics=True, **kw)
    f64 = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision="fp64", **common)
    mix = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision="mixed", **common)
    a, b = mix["coef64"], f64["coef64"]
    nz = np.linalg.norm(b, axis=1) > 0
    per = np.linalg.norm(a - b, axis=1)[nz] / np.linalg.norm(b, axis=1)[nz]
    err = {"global": float(np.linalg.norm(a - b) / np.linalg.norm(b)), "median": float(np.median(per)),
           "p99": float(np.percentile(per, 99)), "max": float(per.max()),
           "iterations_equal": float(np.mean(mix["iterations"][ph.mask] == f64["iterations"][ph.mask]))}
    del f64, mix, a, b
    path = "mixed" if value_mix > value and err["max"] <= 1e-5 else "fp64"

    # ---- e2e: host buffers through the C ABI (pinned host volume)
    pinned = torch.empty(ph.data.shape, dtype=torch.float32, pin_memory=True)
    pinned.numpy()[...] = ph.data
    host_data = pinned.numpy()
    pinned_out = torch.empty((X, Y, Z, K), dtype=torch.float32, pin_memory=True)
    host_out = pinned_out.numpy()
    e2e_t = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(device)
        barrier(world)
        t = time.perf_counter()
        out = shore_fit(host_data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta,
                        small_delta=ph.small_delta, device=device, coefficients_out=host_out, precision=path,
                        **kw)
        dt = time.perf_counter() - t
        if i >= args.warmup:
            e2e_t.append(dt)
    e2e_s = max_over_ranks(sum(e2e_t), world, torch.device("cuda", device))
    e2e_value = world * V * args.steps / e2e_s
    # the drop-in's usual call: a pageable numpy volume and a new output array
    # (the masked rows are gathered into the library's page-locked staging
    # volume on host threads), warm and cold (a new library handle: table
    # set-up, autotuning and allocations included)
    pg_t = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(device)
        barrier(world)
        t = time.perf_counter()
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                  device=device, precision=path, **kw)
        if i >= args.warmup:
            pg_t.append(time.perf_counter() - t)
    pg_host = _abi.last_timing(device)
    pg_s = max_over_ranks(sum(pg_t), world, torch.device("cuda", device))
    # the same with the caller's own (pageable) output array, reused across
    # calls (`coefficients_out`): no fresh pages to fault in
    pre_out = np.empty(ph.data.shape[:3] + (out["coefficients"].shape[-1],), np.float32)
    pre_t = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(device)
        barrier(world)
        t = time.perf_counter()
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                  device=device, precision=path, coefficients_out=pre_out, **kw)
        if i >= args.warmup:
            pre_t.append(time.perf_counter() - t)
    pre_s = max_over_ranks(sum(pre_t), world, torch.device("cuda", device))
    cold_t = []
    for _ in range(2):
        _abi.reset_handle(device)
        torch.cuda.synchronize(device)
        barrier(world)
        t = time.perf_counter()
        shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, big_delta=ph.big_delta, small_delta=ph.small_delta,
                  device=device, precision=path, **kw)
        cold_t.append(time.perf_counter() - t)
    cold_s = max_over_ranks(statistics.median(cold_t), world, torch.device("cuda", device))
    e2e_variants = {"pageable": {"value": world * V * args.steps / pg_s, "unit": "voxels/s",
                                 "ms_per_step": 1e3 * pg_s / args.steps,
                                 "input": "pageable numpy volume, new output array each call",
                                 "ms_host_gather": pg_host.ms_host_gather,
                                 "ms_host_copy_out": pg_host.ms_host_copy_out},
                    "pageable_reused_output": {"value": world * V * args.steps / pre_s, "unit": "voxels/s",
                                               "ms_per_step": 1e3 * pre_s / args.steps,
                                               "input": "pageable numpy volume, the caller's pageable output "
                                                        "array reused (coefficients_out)"},
                    "cold": {"value": world * V / cold_s, "unit": "voxels/s", "ms_per_step": 1e3 * cold_s,
                             "input": "pageable numpy volume on a new library handle (set-up, autotuning and "
                                      "allocations included), median of 2"}}
    # page-locked input: the library reads the masked rows in place (V x N x 4 B) plus the mask
    h2d = V * N * 4 + ph.mask.nbytes
    d2h = out["coefficients"].nbytes

    # ---- the converged-optimum paths on the same volume
    optimum = optimum_block(args, ph, d_data, d_mask, stream, device, world, ms / args.steps)
    # ---- configuration 2's other fits: Tikhonov and the positivity QP
    config2 = config2_block(args, ph, d_data, d_mask, stream, device, world)
    # ---- one volume across the ranks (strong scaling), when there are several
    sharded = sharded_block(args, ph, d_data, stream, device, world) if world > 1 else None
    # ---- fwd+bwd: differentiable fit of 50k voxels
    fwd_bwd = fwd_bwd_block(args, device, world)
    # ---- per-voxel designs (gradient deviation, dropped samples)
    graddev = graddev_block(args, device, world)
    # ---- hypergradient alpha selection pipeline on the same volume
    pipeline = pipeline_block(ph, device, world)

    # ---- roofline of the FISTA kernel
    flops_per_iter = 2 * K * K + 8 * K
    k_ms = statistics.median(kernel_ms)
    it_launch = statistics.median(iters)
    achieved = it_launch * flops_per_iter / (k_ms * 1e-3) / 1e12
    executed = statistics.median(tensor_flops) / (k_ms * 1e-3) / 1e12
    dmma_peak, dfma_peak = fp64_peak_tflops(device)
    traffic = traffic_from_profile(V, statistics.median(parked))
    # warps per CTA the per-table autotuner chose (12 or 16)
    fista_kernel = "k_fista_v3<9," + "/".join(str(w) for w in sorted(warps)) + ">"

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, count, cores, t, stride = cpu_sample_rate(ph, args.cpu_seconds)
        cpu = {"value": rate, "unit": "voxels/s", "cores": cores, "kind": "port",
               "sample": f"every masked voxel at stride {stride} ({count} of {V}; {t:.1f} s), CPU FP64 oracle on all "
                         "host threads"}

    if rank == 0:
        mk_ms = statistics.median(mix_kernel_ms)
        paths = {
            "fp64": {"value": value, "unit": "voxels/s", "ms_per_step": ms / args.steps,
                     "kernel": f"{fista_kernel} (FP64 DMMA mma.sync.m8n8k4), two passes", "kernel_ms": statistics.median(kernel_ms),
                     "gpu_launches": launches},
            "mixed": {"value": value_mix, "unit": "voxels/s", "ms_per_step": ms_mix / args.steps,
                      "speedup_vs_fp64": value_mix / value,
                      "kernel": "k_fista_i8 (tcgen05.mma kind::i8, 36 MMAs 128x80x32 per iteration), two passes",
                      "kernel_ms": mk_ms, "int8_tensor_ops_per_launch": statistics.median(mix_ops),
                      "executed_int8_tops": statistics.median(mix_ops) / (mk_ms * 1e-3) / 1e12 if mk_ms else None,
                      "fp64_rerun_voxels": statistics.median(mix_rerun),
                      "coef_rel_err_vs_fp64": err, "gpu_launches": mix_launches,
                      "clocks": mix_clocks.summary()},
        }
        line = {
            "metric": METRIC, "value": value if path == "fp64" else value_mix, "unit": "voxels/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (ms if path == "fp64" else ms_mix) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if path == "fp64" else "s8 digit-slice products, f64 state",
            "data": "synthetic (seeded CS-DSI multi-tensor phantom, S0 1000, SNR 25)",
            "config": bench_config(ph), "path": path,
            "parallelism": f"{world} independent volume(s), one per GPU",
            "e2e": {"value": e2e_value, "unit": "voxels/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "input": "page-locked volume and output", **e2e_variants},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": dmma_peak, "unit": "TFLOP/s",
                         "frac": (achieved / dmma_peak) if dmma_peak else None, "traffic": traffic,
                         "kernel": fista_kernel, "kernel_ms": k_ms,
                         "kernel_scope": "both passes of the two-pass schedule (to iteration 80, then the "
                                         "parked voxels slowest-first) and the bucket sort between them, "
                                         "timed together with CUDA events",
                         "parked_voxels": statistics.median(parked),
                         "traffic_basis": "ncu per-voxel and per-parked-voxel DRAM bytes of the two passes "
                                          "(fista125k capture) x this run's voxel and parked counts",
                         "flops_per_launch": it_launch * flops_per_iter,
                         "flops_basis": "dense Gram form, executed voxel-iterations x (2K^2 + 8K)",
                         "executed_tensor_flops_per_launch": statistics.median(tensor_flops),
                         "executed_tensor_tflops": executed,
                         "executed_tensor_frac": (executed / dmma_peak) if dmma_peak else None,
                         "peak_source": "FP64 DMMA microbenchmark measured in this run (libcsdpeak); "
                                        f"scalar DFMA measured {dfma_peak:.1f} TFLOP/s" if dmma_peak else None},
            "gpu_launches": launches if path == "fp64" else mix_launches,
            "fwd_bwd": fwd_bwd,
            "graddev": graddev,
            "pipeline": pipeline,
            "paths": paths,
            "optimum": optimum,
            "sharded": sharded,
            "config2": config2,
            "clocks": clocks.summary(),
            "iterations_per_voxel": it_launch / V,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def timed_fits(args, fit, stream, device, world):
    """Device ms per fit over args.steps fits after args.warmup untimed ones
    (CUDA events on the fit stream, max over ranks), with the clock samples."""
    import torch

    for _ in range(args.warmup):
        fit()
    torch.cuda.synchronize(device)
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clocks:
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(args.steps):
            fit()
        e1.record(stream)
        torch.cuda.synchronize(device)
    return max_over_ranks(e0.elapsed_time(e1) / args.steps, world, torch.device("cuda", device)), clocks.summary()


def sharded_block(args, ph, d_data, stream, device: int, world: int) -> dict:
    """The same volume split across the ranks (strong scaling): rank r fits
    its contiguous chunk of the masked voxels (cs_dmri_b200.distributed.shard_mask)
    from the device-resident volume; device time per fit, max over ranks.
    Then one cs_dmri_b200.distributed.fit_sharded call from the host volume -
    fit, gather of every shard's rows to rank 0, reassembly - on the host
    clock."""
    import torch

    from cs_dmri_b200 import shore_fit_device
    from cs_dmri_b200.distributed import fit_sharded, shard_mask

    rank = int(os.environ.get("RANK", "0"))
    V = int(ph.mask.sum())
    local = torch.from_numpy(shard_mask(ph.mask, rank, world)).to(f"cuda:{device}")
    kw = dict(fit_kwargs(), big_delta=ph.big_delta, small_delta=ph.small_delta, device=device)

    def fit():
        return shore_fit_device(d_data, local, ph.bvals, ph.bvecs, stream=stream, **kw)

    ms_step, clk = timed_fits(args, fit, stream, device, world)
    torch.cuda.synchronize(device)
    barrier(world)
    t = time.perf_counter()
    fit_sharded(ph.data, ph.bvals, ph.bvecs, ph.mask, **kw)
    dt = max_over_ranks(time.perf_counter() - t, world, torch.device("cuda", device))
    return {"metric": "voxels/s of one volume across all ranks", "scaling": "strong", "value": V / (ms_step * 1e-3),
            "unit": "voxels/s", "ms_per_step": ms_step, "voxels_per_rank": V // world, "clocks": clk,
            "fit_sharded_host_s": dt, "fit_sharded_voxels_per_s": V / dt}


def config2_block(args, ph, d_data, d_mask, stream, device: int, world: int) -> dict:
    """The brain-sized volume's other two fits of configuration 2, device
    buffers in and out:
      l2      Tikhonov, lambda_n = lambda_l = 0.05: c = P s with the solution
              operator P = H^-1 M^T (built once per table from the Cholesky
              factor of H, src/solver/tikhonov.rs:26-76), one FP64 DMMA
              product per 8 voxels (k_rhs_dmma with P in place of M^T);
              algorithmic work 2 N K FLOP and 4 N + 8 K bytes per voxel;
      nonneg  the amplitude-positivity QP (Goldfarb-Idnani in Gram form,
              k_icls_gram: the constraint values carried through W^T W),
              credited with the reference's arithmetic, iterations x
              (2 m K + 2 K^2) FLOP with m = 321 constraints (the scan it no
              longer runs included), so the figure compares with the
              recomputing form."""
    from cs_dmri_b200 import _abi, shore_fit_device

    V = int(ph.mask.sum())
    N, K, m = ph.data.shape[-1], 72, 321
    base = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, device=device, radial_order=6, zeta=700.0)
    out = {}
    for name, kw in (("l2", dict(regularization="l2", lambda_n=0.05, lambda_l=0.05)),
                     ("nonneg", dict(regularization="nonneg"))):
        def fit():
            return shore_fit_device(d_data, d_mask, ph.bvals, ph.bvecs, stream=stream, **base, **kw)
        ms_step, clk = timed_fits(args, fit, stream, device, world)
        coef, res = fit()
        t = _abi.last_timing(device)
        blk = {"value": world * V / (ms_step * 1e-3), "unit": "voxels/s", "ms_per_step": ms_step, "clocks": clk}
        if name == "l2":
            k_ms = t.ms_rhs  # the operator product is the whole solve
            flops = 2.0 * N * K * V
            byts = (4.0 * N + 8.0 * K) * V
            blk.update({"kernel": "k_rhs_dmma<72> with the Tikhonov operator (FP64 DMMA)", "kernel_ms": k_ms,
                        "achieved_tflops": flops / (k_ms * 1e-3) / 1e12,
                        "achieved_gbs": byts / (k_ms * 1e-3) / 1e9})
        else:
            k_ms = t.ms_solve_kernel
            it = res.total_iterations / V
            flops = res.total_iterations * (2.0 * m * K + 2.0 * K * K)
            blk.update({"kernel": "k_icls_gram (FP64, warp per voxel, Gram form)", "kernel_ms": k_ms,
                        "iterations_per_voxel": it,
                        "reference_equivalent_tflops": flops / (k_ms * 1e-3) / 1e12})
        out[name] = blk
    return out


def optimum_block(args, ph, d_data, d_mask, stream, device: int, world: int, fp64_ms: float) -> dict:
    """The LASSO optimum itself (precision "mixed-kkt": TF32 tensor-core FISTA
    iterations find the support, an FP64 active-set polish solves on it and
    certifies every voxel by its KKT conditions) against three FP64 GPU
    references on the same volume:
      fp64       the reference stopping rule (tol 1e-6) - the parity path,
                 whose output is not the optimum;
      fp64-kkt   the same support identification with FP64 iterations;
      fp64-tight the reference FISTA with tol 1e-9 and max_iter 20000, the
                 plain FP64 path run far enough to approach the optimum.
    Errors are per-voxel relative L2 against the certified optimum, whole
    volume; KKT residuals in the form of the reference's
    tests/common/mod.rs:127-153."""
    import torch

    from cs_dmri_b200 import _abi, shore_fit, shore_fit_device

    V = int(ph.mask.sum())
    base = dict(fit_kwargs(), big_delta=ph.big_delta, small_delta=ph.small_delta, device=device)
    tight = dict(base, tol=1e-9, max_iter=20000)

    def dev(precision, kw):
        return lambda: shore_fit_device(d_data, d_mask, ph.bvals, ph.bvecs, stream=stream, precision=precision,
                                        **kw)

    out = {"metric": "converged-optimum L1-fit voxels/s", "unit": "voxels/s", "workload": f"{WORKLOAD}: {V} voxels",
           "certificate": "every off-support |M_j^T (M c - s)| / n <= alpha (1 + 1e-9), signs consistent on the "
                          "support"}
    ms_kkt, clk = timed_fits(args, dev("mixed-kkt", base), stream, device, world)
    t = _abi.last_timing(device)
    out["mixed_kkt"] = {"value": world * V / (ms_kkt * 1e-3), "ms_per_step": ms_kkt,
                        "speedup_vs_fp64_reference_rule": fp64_ms / ms_kkt,
                        "ms_iterate": t.ms_kkt_iterate, "ms_polish": t.ms_kkt_polish,
                        "ms_fallback": t.ms_kkt_fallback, "ms_rhs": t.ms_rhs,
                        "fallback_voxels": t.kkt_fallback_voxels, "uncertified_voxels": t.kkt_uncertified,
                        "polish_rounds_per_voxel": t.kkt_rounds / V, "kkt_max": t.kkt_max,
                        "tf32_tensor_tflops_executed": t.tf32_tensor_flops / (t.ms_kkt_iterate * 1e-3) / 1e12
                        if t.ms_kkt_iterate else None,
                        "support_iterations": t.kkt_iterations,
                        "autotune_ms_16_24_32_48": list(t.kkt_tune_ms),
                        "polish_supports_past_32": int(t.kkt_overflow),
                        "kernels": "k_fista_tf32 (tcgen05.mma kind::tf32, 128 voxels x 80 x 72 per iteration), "
                                   "k_l1_polish (FP64, warp per voxel)",
                        "clocks": clk}
    ms_f, clk = timed_fits(args, dev("fp64-kkt", base), stream, device, world)
    t = _abi.last_timing(device)
    out["fp64_kkt"] = {"value": world * V / (ms_f * 1e-3), "ms_per_step": ms_f, "ms_iterate": t.ms_kkt_iterate,
                       "ms_polish": t.ms_kkt_polish, "uncertified_voxels": t.kkt_uncertified, "clocks": clk}
    targs = argparse.Namespace(warmup=1, steps=max(1, min(args.steps, 3)))
    ms_t, clk = timed_fits(targs, dev("fp64", tight), stream, device, world)
    out["fp64_tight"] = {"value": world * V / (ms_t * 1e-3), "ms_per_step": ms_t, "tol": 1e-9, "max_iter": 20000,
                         "steps": targs.steps, "clocks": clk}
    out["mixed_kkt"]["speedup_vs_fp64_kkt"] = ms_f / ms_kkt
    out["mixed_kkt"]["speedup_vs_fp64_tight"] = ms_t / ms_kkt

    # errors against the certified optimum, whole volume (FP64 outputs)
    common = dict(return_coef64=True, diagnostics=True)
    opt = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision="mixed-kkt", **common, **base)
    ok = opt["converged"]
    c_opt = opt["coef64"]
    nrm = np.linalg.norm(c_opt, axis=1)
    sel = ok & (nrm > 0)

    def errs(c):
        r = np.linalg.norm(c[sel] - c_opt[sel], axis=1) / nrm[sel]
        return {"median": float(np.median(r)), "p99": float(np.percentile(r, 99)), "max": float(r.max()),
                "frac_above_1e-5": float(np.mean(r > 1e-5))}

    out["certified_fraction"] = float(ok.mean())
    out["fp64"] = {"value": world * V / (fp64_ms * 1e-3), "ms_per_step": fp64_ms,
                   "note": "the FP64 path of paths.fp64 (reference stopping rule)"}
    for name, kw, prec in (("fp64_kkt", base, "fp64-kkt"), ("fp64", base, "fp64"), ("fp64_tight", tight, "fp64")):
        res = shore_fit(ph.data, ph.bvals, ph.bvecs, ph.mask, precision=prec, **common, **kw)
        out[name]["coef_rel_err_vs_optimum"] = errs(res["coef64"])
        del res
    del opt, c_opt
    return out


def fwd_bwd_block(args, device: int, world: int) -> dict:
    """Differentiable fit (forward + adjoint) on 50,000 voxels of the same
    generator, radial order 6.  One step: the fit (L1 at alpha 0.01, or
    Tikhonov at lambda 0.05), RTOP and the ODF on the 362-vertex geodesic
    sphere, then backward to the float32 signals and the float64
    hyper-parameters, every kernel in libcsdshore.so.  CUDA events on the
    stream the calls run on; max over ranks.  Inputs stay resident (52 MB of
    signals; the step's own buffers exceed L2 several times over)."""
    import torch

    from cs_dmri_b200.autograd import DifferentiableShore
    from cs_dmri_b200.phantom import make_phantom

    ph = make_phantom(FWD_BWD_GRID, seed=4)
    S = torch.from_numpy(ph.data.reshape(-1, ph.data.shape[-1])).to(f"cuda:{device}")
    V = S.shape[0]
    out = {"metric": "fwd+bwd voxels/s", "workload": f"diff50k: {V} voxels, radial order 6, N = {S.shape[1]}",
           "unit": "voxels/s", "dtype": "f64 (signals f32)",
           "step": "fit + RTOP + ODF (362 directions) forward, backward to signals and the hyper-parameter"}
    for reg in ("l1", "l2"):
        m = DifferentiableShore(ph.bvals, ph.bvecs, regularization=reg, big_delta=ph.big_delta,
                                small_delta=ph.small_delta, device=device)

        def step(bwd: bool):
            s = S.detach().requires_grad_(bwd)
            if reg == "l1":
                a = torch.tensor(0.01, dtype=torch.float64, device=S.device, requires_grad=bwd)
                c = m.fit(s, a)
            else:
                a = torch.tensor(0.05, dtype=torch.float64, device=S.device, requires_grad=bwd)
                c = m.fit(s, lambda_n=a, lambda_l=a)
            loss = m.rtop(c).sum() + 1e-3 * m.odf(c).square().sum()
            if bwd:
                loss.backward()

        res = {}
        for bwd in (False, True):
            for _ in range(args.warmup):
                step(bwd)
            torch.cuda.synchronize(device)
            barrier(world)
            st = torch.cuda.current_stream(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(args.steps):
                step(bwd)
            e1.record(st)
            torch.cuda.synchronize(device)
            ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, torch.device("cuda", device))
            res["fwd_bwd" if bwd else "fwd"] = ms
        block = {"value": world * V / (res["fwd_bwd"] * 1e-3), "ms_per_step": res["fwd_bwd"],
                 "fwd_value": world * V / (res["fwd"] * 1e-3), "fwd_ms_per_step": res["fwd"],
                 "fwd_bwd_over_fwd": res["fwd_bwd"] / res["fwd"]}
        if reg == "l1":
            out.update(block)
            out["solver"] = "L1 FISTA, alpha 0.01 (tol 1e-6), implicit differentiation on the support"
        else:
            out["l2"] = dict(block, solver="Tikhonov, lambda_n = lambda_l = 0.05, adjoint as one product with H^-1")
    return out


def graddev_block(args, device: int, world: int) -> dict:
    """L1 fit on a design per voxel: 300,000 voxels of the phantom, each with
    its own gradient-deviation tensor (I + N(0, 0.02)) and 0-15 % of its
    samples dropped, radial order 8 (K = 145), alpha 0.01: the reference's
    FISTA (`value`), and the certified optimum of each voxel's design
    (precision "fp64-kkt": 32 FISTA iterations, the polish on the voxel's own
    Gram matrix, the KKT certificate), and its mixed-precision form
    ("mixed-kkt": the Lanczos estimate and the support iterations in FP32 on
    the hi plane of G_v, the polish in FP64 on hi + lo) with its error per
    output (coefficients, RTOP, GFA) against the FP64 certified optimum.  CUDA events on the fit stream, max
    over ranks; min(steps, 3) timed steps (each builds 300k Gram matrices of
    145 x 145)."""
    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200.graddev import graddev_phantom, shore_fit_graddev

    S, bvals, bvecs, T, keep, big, small = graddev_phantom(GRADDEV_VOXELS, seed=3)
    dev = f"cuda:{device}"
    St, Tt, Kt = (torch.from_numpy(a).to(dev) for a in (S, T, keep))
    steps = max(1, min(args.steps, 3))

    def timed(precision):
        kw = dict(alpha=0.01, radial_order=8, big_delta=big, small_delta=small, device=device, precision=precision)
        out = shore_fit_graddev(St, bvals, bvecs, Tt, Kt, **kw)  # one untimed fit: each is a second of work
        torch.cuda.synchronize(device)
        barrier(world)
        st = torch.cuda.current_stream(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            out = shore_fit_graddev(St, bvals, bvecs, Tt, Kt, **kw)
        e1.record(st)
        torch.cuda.synchronize(device)
        return max_over_ranks(e0.elapsed_time(e1) / steps, world, torch.device("cuda", device)), out

    ms, out = timed("fp64")
    it = float(out["iterations"].double().mean())
    ms_k, out_k = timed("fp64-kkt")
    t = _abi.last_timing(device)
    ms_m, out_m = timed("mixed-kkt")
    t_m = _abi.last_timing(device)
    errors = graddev_output_errors(out_k["coefficients"], out_m["coefficients"], device)
    return {"metric": "per-voxel-design L1-fit voxels/s", "value": world * GRADDEV_VOXELS / (ms * 1e-3),
            "unit": "voxels/s", "ms_per_step": ms, "steps": steps,
            "workload": f"graddev300k: {GRADDEV_VOXELS} voxels, radial order 8 (K = 145), N = {S.shape[1]}, "
                        "deviation tensor and 0-15 % dropped samples per voxel",
            "dtype": "f64", "iterations_per_voxel": it,
            "kkt": {"value": world * GRADDEV_VOXELS / (ms_k * 1e-3), "ms_per_step": ms_k,
                    "speedup_vs_reference_rule": ms / ms_k, "uncertified_voxels": t.kkt_uncertified,
                    "polish_rounds_per_voxel": t.kkt_rounds / GRADDEV_VOXELS,
                    "support_iterations": t.kkt_iterations,
                    "autotune_ms_16_24_32_48": list(t.kkt_tune_ms),
                    "certified_fraction": float(out_k["converged"].double().mean())},
            "mixed_kkt": {"value": world * GRADDEV_VOXELS / (ms_m * 1e-3), "ms_per_step": ms_m,
                          "speedup_vs_reference_rule": ms / ms_m, "speedup_vs_fp64_kkt": ms_k / ms_m,
                          "uncertified_voxels": t_m.kkt_uncertified,
                          "polish_rounds_per_voxel": t_m.kkt_rounds / GRADDEV_VOXELS,
                          "support_iterations": t_m.kkt_iterations,
                          "autotune_ms_16_24_32_48": list(t_m.kkt_tune_ms),
                          "certified_fraction": float(out_m["converged"].double().mean()),
                          "dtype": "f32 Lanczos and support iterations, f64 polish and certificate",
                          "error_vs_fp64_kkt": errors}}


def graddev_output_errors(ref, got, device: int) -> dict:
    """Per-output error of a per-voxel-design fit (radial order 8, zeta 700)
    against an FP64 one: coefficients (per-voxel relative L2), RTOP (relative)
    and GFA (absolute, on the 181-direction hemisphere)."""
    import ctypes as C

    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200._core import shore_odf_peaks

    def stats(e):
        e = np.asarray(e, np.float64)
        e = e[np.isfinite(e)]
        return {"median": float(np.median(e)), "p99": float(np.quantile(e, 0.99)), "max": float(e.max())}

    a, b = ref.double().contiguous(), got.double().contiguous()
    rel = (torch.linalg.norm(a - b, dim=1) / torch.linalg.norm(a, dim=1).clamp_min(1e-300)).cpu().numpy()
    lib = _abi.load()
    rt = []
    for c in (a, b):
        r = torch.empty(c.shape[0], dtype=torch.float64, device=c.device)
        err = C.create_string_buffer(1024)
        _abi.check(lib.csd_shore_rtop_device(_abi.handle(device), 8, 700.0, c.data_ptr(), c.shape[0], r.data_ptr(),
                                             None, err, len(err)), err)
        rt.append(r)
    torch.cuda.synchronize(device)
    ra, rb = rt[0].cpu().numpy(), rt[1].cpu().numpy()
    rtop = np.abs(ra - rb) / np.maximum(np.abs(ra), 1e-300)
    gfa = [shore_odf_peaks(c.cpu().numpy().astype(np.float32).reshape(-1, 1, 1, c.shape[1]), 8, 700.0,
                           npeaks=1, device=device)["gfa"].ravel() for c in (a, b)]
    return {"coefficients_rel_l2": stats(rel), "rtop_rel": stats(rtop), "gfa_abs": stats(np.abs(gfa[0] - gfa[1]))}


def pipeline_block(ph, device: int, world: int) -> dict:
    """The hypergradient pipeline on the brain-sized volume: per-voxel alpha by
    8 Rprop steps on the hypergradient of a held-out 10 % of the samples, the
    final fit on every sample, 3 peaks + GFA, RTOP and MSD (host volumes in
    and out).  One untimed run, then one run on the host clock (it includes
    the host copies); the reference's own selections (L2-anchored, path-BIC)
    and the fixed alpha are scored on the same held-out samples in that run."""
    import torch

    from cs_dmri_b200.hyper import select_alpha_hypergradient

    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, device=device)
    select_alpha_hypergradient(ph.data, ph.bvals, ph.bvecs, ph.mask, compare_reference=False, **kw)
    torch.cuda.synchronize(device)
    barrier(world)
    t = time.perf_counter()
    out = select_alpha_hypergradient(ph.data, ph.bvals, ph.bvecs, ph.mask, compare_reference=False, **kw)
    torch.cuda.synchronize(device)
    dt = max_over_ranks(time.perf_counter() - t, world, torch.device("cuda", device))
    comp = select_alpha_hypergradient(ph.data, ph.bvals, ph.bvecs, ph.mask, compare_reference=True,
                                      **kw)["comparison"]
    V = int(ph.mask.sum())
    return {"metric": "hypergradient-pipeline voxels/s", "value": world * V / dt, "unit": "voxels/s",
            "seconds": dt, "workload": f"{WORKLOAD}: {V} voxels, 8 hypergradient steps, final fit, 3 peaks, "
                                       "GFA, RTOP, MSD (host volumes in and out)",
            "heldout_error_median": comp,
            "alpha_median": float(np.median(out["alpha"][ph.mask]))}


# ------------------------------------------------------------------ profiling cases
#
# Small, fixed workloads that run one pass of a kernel family, for profiling
# under ncu (a few launches of each kernel of interest, a few hundred MB on
# the device at most): python bench.py --profile-case NAME.

def case_graddev2k() -> None:
    import torch

    from cs_dmri_b200.graddev import graddev_phantom, shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = graddev_phantom(2000, seed=3)
    out = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, radial_order=8, big_delta=big, small_delta=small)
    torch.cuda.synchronize()
    print("graddev2k: mean iterations", float(out["iterations"].double().mean()))


def case_graddev2k_mixed() -> None:
    import torch

    from cs_dmri_b200.graddev import graddev_phantom, shore_fit_graddev
    S, bvals, bvecs, T, keep, big, small = graddev_phantom(2000, seed=3)
    out = shore_fit_graddev(S, bvals, bvecs, T, keep, alpha=0.01, radial_order=8, big_delta=big, small_delta=small,
                            precision="mixed-kkt")
    torch.cuda.synchronize()
    print("graddev2k-mixed: certified fraction", float(out["converged"].double().mean()))


def case_diff50k() -> None:
    import torch

    from cs_dmri_b200.autograd import DifferentiableShore
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((50, 50, 20), seed=4)
    S = torch.from_numpy(ph.data.reshape(-1, ph.data.shape[-1])).cuda().requires_grad_(True)
    m = DifferentiableShore(ph.bvals, ph.bvecs, big_delta=ph.big_delta, small_delta=ph.small_delta)
    a = torch.tensor(0.01, dtype=torch.float64, device="cuda", requires_grad=True)
    c = m.fit(S, a)
    (m.rtop(c).sum() + 1e-3 * m.odf(c).square().sum()).backward()
    torch.cuda.synchronize()
    print("diff50k: d loss / d alpha", float(a.grad))


def case_peaks108k() -> None:
    from cs_dmri_b200._core import shore_odf_peaks
    rng = np.random.default_rng(1)
    vol = rng.normal(size=(60, 60, 30, 72)).astype(np.float32)
    vol[..., 0] = np.abs(vol[..., 0]) + 5.0
    out = shore_odf_peaks(vol, 6, 700.0)
    print("peaks108k: mean GFA", float(out["gfa"].mean()))


def case_fista125k() -> None:
    """A fixed-alpha fit of a 50^3 phantom (125,000 voxels, K = 72) through the
    device entry point: enough voxels per FISTA slot for the two-pass
    schedule (pass 1 to iteration 80, bucket sort, pass 2).  A first fit
    (gradient-table set-up, autotuning) runs outside the NVTX range."""
    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200._core import shore_fit_device
    from cs_dmri_b200.phantom import make_phantom
    ph = make_phantom((50, 50, 50), seed=6)
    d = torch.from_numpy(ph.data).cuda()
    m = torch.from_numpy(ph.mask).cuda()
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01)
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("fista125k")
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    t = _abi.last_timing(0)
    print(f"fista125k: solve {t.ms_solve_kernel:.3f} ms, parked {t.fista_parked} of {int(ph.mask.sum())} voxels")


def case_kkt64k() -> None:
    """The converged-optimum fit (precision "mixed-kkt") of the 40^3 phantom
    (64,000 voxels, K = 72) through the device entry point, 32 support
    iterations: one launch each of k_fista_tf32 and the two k_l1_polish passes
    per fit.  A first fit (set-up) runs before the
    measured one."""
    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200._core import shore_fit_device
    from cs_dmri_b200.phantom import config_phantom
    ph = config_phantom("grid64k")
    d = torch.from_numpy(ph.data).cuda()
    m = torch.from_numpy(ph.mask).cuda()
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, alpha_mode="fixed", alpha=0.01,
              precision="mixed-kkt")
    _abi.set_option(_abi.OPT_KKT_ITERATIONS, 32)  # a fixed count: no autotuning batches in the launch list
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    torch.cuda.synchronize()
    t = _abi.last_timing(0)
    print(f"kkt64k: iterate {t.ms_kkt_iterate:.3f} ms, polish {t.ms_kkt_polish:.3f} ms, "
          f"fallback voxels {t.kkt_fallback_voxels}, uncertified {t.kkt_uncertified}")


def _case_grid64k(name: str, **fit_kw) -> None:
    """One fit of the 40^3 phantom (64,000 voxels, K = 72) through the device
    entry point after a set-up fit of the same kind."""
    import torch

    from cs_dmri_b200 import _abi
    from cs_dmri_b200._core import shore_fit_device
    from cs_dmri_b200.phantom import config_phantom
    ph = config_phantom("grid64k")
    d = torch.from_numpy(ph.data).cuda()
    m = torch.from_numpy(ph.mask).cuda()
    kw = dict(big_delta=ph.big_delta, small_delta=ph.small_delta, **fit_kw)
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    shore_fit_device(d, m, ph.bvals, ph.bvecs, **kw)
    torch.cuda.synchronize()
    t = _abi.last_timing(0)
    print(f"{name}: solve kernel {t.ms_solve_kernel:.3f} ms, right-hand side {t.ms_rhs:.3f} ms, "
          f"total {t.ms_total:.3f} ms")


def case_icls64k() -> None:
    """The amplitude-positivity QP (k_icls) on the 40^3 phantom."""
    _case_grid64k("icls64k", regularization="nonneg")


def case_tikhonov64k() -> None:
    """The Tikhonov fit (lambda_n = lambda_l = 0.05): one k_rhs_dmma launch
    with the solution operator on the 40^3 phantom."""
    _case_grid64k("tikhonov64k", regularization="l2", lambda_n=0.05, lambda_l=0.05)


PROFILE_CASES = {"graddev2k": case_graddev2k, "graddev2k-mixed": case_graddev2k_mixed, "diff50k": case_diff50k, "peaks108k": case_peaks108k,
                 "fista125k": case_fista125k, "kkt64k": case_kkt64k, "icls64k": case_icls64k,
                 "tikhonov64k": case_tikhonov64k}


def launch_ranks(args) -> int:
    """`--gpus N` without a launcher: run this script under torchrun with N
    ranks on this node (rendezvous on 127.0.0.1); rank 0 prints the line."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.profile_case:
        PROFILE_CASES[args.profile_case]()
        return 0
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args)
    select_workload(args.workload)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
