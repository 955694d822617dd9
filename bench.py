#!/usr/bin/env python
"""Throughput of the fused D3Q19 TRT stream-collide step on B200.

Workload (one "step" = one fused pull-stream + TRT collide pass over the
grid): periodic D3Q19 Taylor-Green vortex, 256^3 nodes, TRT magic parameter
1/4, nu = 0.01, u0 = 0.05, rho0 = 1, populations in HBM (default storage:
FP32 deviations f - w_q; --storage picks f64 | f32 | f32dev | f16dev |
bf16dev).  Moments are written at the check cadence (every 100 steps), not
every step.  Each population buffer (1.27 GB in FP32) is larger than the
126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W --storage S]
  python bench.py --impl reference ...   # the reference's CPU path (oracle port)

Prints one JSON line (rank 0).  `value` is whole-job MLUPS with populations
resident in HBM; `e2e` is the same metric through the public API with the
initial populations copied from pinned host memory and the final moments
read back inside the timed region.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS & % HBM roofline per lattice/precision; time-to-steady vs plain"
N_GRID = 256
NU, LAMBDA, U0 = 0.01, 0.25, 0.05
CHECK_EVERY = 100
FALLBACK_HBM_GBS = 6650.0

STORAGES = {
    # name: (torch dtype name, deviation, bytes per population, kb dtype label)
    "f64": ("float64", False, 8, "f64"),
    "f32": ("float32", False, 4, "f32"),
    "f32dev": ("float32", True, 4, "f32 (f-w)"),
    "f16dev": ("float16", True, 2, "f16 (f-w)"),
    "bf16dev": ("bfloat16", True, 2, "bf16 (f-w)"),
    "f16dev_sr": ("float16", True, 2, "f16 (f-w), stochastic rounding"),
    "bf16dev_sr": ("bfloat16", True, 2, "bf16 (f-w), stochastic rounding"),
}
SR_STORAGES = {"f16dev_sr", "bf16dev_sr"}


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(storage):
    """DRAM bytes per launch of the fused TRT kernel from the committed ncu
    summary (profiles/d3q19_trt_tgv_traffic.txt: lines `storage bytes`)."""
    p = ROOT / "profiles" / "d3q19_trt_tgv_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == storage and not line.startswith("#"):
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    (nvidia_ml_py) every 10 ms on the GPU with the CUDA device's PCI bus id,
    else nvidia-smi every 100 ms.  start() returns once the first sample is
    in, so the samples cover the whole timed region.  Read-only queries."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []  # (sm_mhz, max_mhz, reason bits) from NVML
        self.t = None
        self.nvml = None
        self.stop_flag = threading.Event()
        self.first = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h):
        getr = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_flag.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), smax, getr(h)))
            except Exception:
                pass
            self.first.set()
            self.stop_flag.wait(0.01)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = nv
            self.t = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.t.start()
            self.first.wait(5)
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(5)
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.t.join(timeout=5)
            sm = [s[0] for s in self.samples]
            bits = 0
            for s in self.samples:
                bits |= int(s[2])
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": self.samples[0][1] if self.samples else None,
                    "reasons": sorted(k for k, b in self.REASONS.items() if bits & b),
                    "samples": len(sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def dist_setup(gpus):
    import torch
    import torch.distributed as dist
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    if world > 1:
        from datetime import timedelta
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- CPU arm --

# Precision of the reference's CPU path that a GPU storage is timed against:
# FP64 for FP64; the reference's T = Float32 path (its narrowest) for the
# FP32 storages and the 16-bit deviation storages.
CPU_PRECISION = {"f64": "f64", "f32": "f32", "f32dev": "f32", "f16dev": "f32", "bf16dev": "f32",
                 "f16dev_sr": "f32", "bf16dev_sr": "f32"}


def tgv_config(n, storage, world):
    """The `config` of the TGV bench line, shared by the GPU and reference arms."""
    return {"workload": f"D3Q19 TRT periodic Taylor-Green {n}^3, Lambda=1/4, nu={NU}, "
                        f"u0={U0}, rho0=1", "grid": [n, n, n], "storage": storage,
            "moments": f"written every {CHECK_EVERY} steps",
            "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"replicas x{world}" if world > 1 else "none"}


def cpu_reference_mlups(n, steps_cap, budget_s, threads, precision="f32", warmup=1):
    """The oracle port (C restatement of the reference's CPU path, OpenMP) on
    a periodic n^3 D3Q19 TRT Taylor-Green vortex, in FP64 or in the
    reference's Float32 arithmetic.  Returns (MLUPS, steps, seconds, nz) timed
    after `warmup` untimed steps; the z extent is cut to keep one step near
    budget_s/steps_cap seconds on slow hosts (the first warm-up step sizes
    it)."""
    import numpy as np
    import __graft_entry__ as graft
    orc = graft.load_oracle()
    pkg = graft.load_package()
    orc.set_threads(threads)
    dt_np = np.float64 if precision == "f64" else np.float32
    step = orc.fused_trt_3d if precision == "f64" else orc.fused_trt_3d_f32
    nz = n
    plane = pkg.drivers.taylor_green_3d_populations(n, U0, Nz=1).astype(dt_np)
    f = np.ascontiguousarray(np.broadcast_to(plane, (19, nz, n, n)))
    g = np.empty_like(f)
    sp, sm = orc.trt_rates(NU, LAMBDA)
    t0 = time.perf_counter()
    step(g, f, None, None, sp, sm, (1, 1, 1))
    t1 = time.perf_counter() - t0
    per_step_budget = budget_s / max(1, steps_cap)
    if t1 > per_step_budget and nz > 8:
        nz = max(8, int(nz * per_step_budget / t1))
        f = np.ascontiguousarray(np.broadcast_to(plane, (19, nz, n, n)))
        g = np.empty_like(f)
    for _ in range(max(0, warmup - 1) if nz == n else max(1, warmup)):
        step(g, f, None, None, sp, sm, (1, 1, 1))
        f, g = g, f
    steps = 0
    t0 = time.perf_counter()
    while steps < steps_cap:
        step(g, f, None, None, sp, sm, (1, 1, 1))
        f, g = g, f
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return steps * n * n * nz / dt / 1e6, steps, dt, nz


def _cpu_sample(n, nz, steps, warmup, precision, threads):
    arith = "FP64" if precision == "f64" else "FP32 (the reference's T=Float32 path)"
    return (f"periodic D3Q19 TRT Taylor-Green {n}x{n}x{nz} (z cut to bound the run), {steps} "
            f"steps after {warmup} warm-up, {arith}, C restatement of the reference CPU path "
            f"(Julia reference not runnable here), OpenMP {threads} threads")


def run_reference(args):
    # the reference arm runs no collectives: rank 0 times the CPU path, the
    # other ranks of a torchrun launch exit at once without joining a group
    rank, world = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1)
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    prec = CPU_PRECISION[args.storage]
    warmup = max(1, args.warmup)
    mlups, steps, dt, nz = cpu_reference_mlups(N_GRID, max(1, args.steps), 150.0, threads,
                                               prec, warmup)
    sample = _cpu_sample(N_GRID, nz, steps, warmup, prec, threads)
    line = {"impl": "reference", "metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS",
            "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
            "ms_per_step": round(1e3 * dt / steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": prec, "data": "synthetic",
            "config": tgv_config(N_GRID, args.storage, world),
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm --

def run_gpu(args):
    import torch
    import __graft_entry__ as graft

    rank, world, local = dist_setup(args.gpus)
    pkg = graft.load_package()
    pkg._lib.load()
    pkg.set_trt3d_variant(args.trt_variant)
    dev = torch.device("cuda", torch.cuda.current_device())
    tname, deviation, bpp, dlabel = STORAGES[args.storage]
    dtype = getattr(torch, tname)
    n = args.grid
    nodes = n ** 3
    fd = torch.float64 if dtype == torch.float64 else torch.float32

    # initial populations: one z-plane on the host, extruded on the device
    plane = torch.from_numpy(pkg.drivers.taylor_green_3d_populations(n, U0, Nz=1)).to(dev)
    f64 = plane.expand(19, n, n, n)
    f_in = torch.empty((19, n, n, n), dtype=dtype, device=dev)
    if dtype == torch.float64 and not deviation:
        f_in.copy_(f64)
    else:
        pkg.convert_populations(f_in, _extrude(plane, n), dst_deviation=deviation)
    del f64
    f_out = torch.empty_like(f_in)
    mom = [torch.empty((n, n, n), dtype=fd, device=dev) for _ in range(4)]
    none4 = (None, None, None, None)
    stream = torch.cuda.current_stream()

    sr = args.storage in SR_STORAGES

    def step(s, fi, fo):
        m = mom if (s + 1) % CHECK_EVERY == 0 else none4
        pkg.fused_trt_step_3d_(fo, fi, *m, None, n, n, n, NU, LAMBDA, periodic=(1, 1, 1),
                               deviation=deviation, stochastic_rounding=sr)

    a, b = f_in, f_out
    for s in range(args.warmup):
        step(s, a, b)
        a, b = b, a
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for s in range(args.steps):
        step(s, a, b)
        a, b = b, a
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = world * nodes * args.steps / (ms_max * 1e-3) / 1e6
    kernel_ms = ms / args.steps

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty((19, n, n, n), dtype=dtype, pin_memory=True)
        host.copy_(a)
        out_host = [torch.empty((n, n, n), dtype=fd, pin_memory=True) for _ in range(4)]
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        a.copy_(host, non_blocking=True)
        for s in range(args.steps):
            last = s == args.steps - 1
            m = mom if last else none4
            pkg.fused_trt_step_3d_(b, a, *m, None, n, n, n, NU, LAMBDA, periodic=(1, 1, 1),
                                   deviation=deviation, stochastic_rounding=sr)
            a, b = b, a
        for h, d in zip(out_host, mom):
            h.copy_(d, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ems = max_over_ranks(e0.elapsed_time(e1), world)
        h2d = host.numel() * host.element_size()
        d2h = sum(t.numel() * t.element_size() for t in out_host)
        e2e = {"value": round(world * nodes * args.steps / (ems * 1e-3) / 1e6, 1), "unit": "MLUPS",
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "note": (f"timed: pinned host->device copy of the initial populations, {args.steps} "
                        "fused steps through the public API, device->host copy of rho,u; bytes "
                        "per step = total / steps")}
        del host, out_host

    peak, peak_kind = hbm_peak()
    alg_bytes = 2 * 19 * bpp * nodes
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    traffic = traffic_per_launch(args.storage)

    line = None
    if rank == 0:
        cpu = cpu64 = None
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            prec = CPU_PRECISION[args.storage]
            mlups, steps, dt, nz = cpu_reference_mlups(n, 20, 15.0, threads, prec, 3)
            cpu = {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                   "sample": _cpu_sample(n, nz, steps, 3, prec, threads) + f", {dt:.1f} s"}
            if prec != "f64" and not args.no_extra:
                mlups, steps, dt, nz = cpu_reference_mlups(n, 20, 15.0, threads, "f64", 3)
                cpu64 = {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads,
                         "kind": "port",
                         "sample": _cpu_sample(n, nz, steps, 3, "f64", threads) + f", {dt:.1f} s"}
        extra = None
        if not args.no_extra and world == 1:
            extra = {"cpu_baseline_f64": cpu64,
                     "tgv_config2_precisions": bench_tgv_precisions(pkg, n, 2000),
                     "cavity2d_config1": bench_cavity2d(pkg, steps=20000),
                     "natconv_config4": bench_natconv(pkg, 512, 1e5, 2000)[0],
                     "d2q9_fused_4096": bench_d2q9_large(pkg),
                     "unfused_paths": bench_unfused_paths(pkg),
                     "thermal_guo_paths": bench_thermal_guo_paths(pkg),
                     "batch_config3_short": bench_batch(pkg, max_steps=2000, check_every=100,
                                                        autotune=True)}
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dlabel,
            "data": "synthetic",
            "config": tgv_config(n, args.storage, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "algorithmic_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clocks,
            "extra": extra,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------- other workloads --

def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def bench_tgv_precisions(pkg, n=N_GRID, steps=2000):
    """Config 2 accuracy and speed per storage: periodic D3Q19 TRT
    Taylor-Green n^3, Lambda=1/4, nu=0.01, u0=0.05, `steps` steps.  Reports
    MLUPS, the HBM roofline fraction and the relative L2 / max velocity
    error against the FP64 run and against exp(-2 nu k^2 t)."""
    import numpy as np
    import torch
    k = 2 * math.pi / n
    decay = math.exp(-2 * NU * k * k * steps)
    x = torch.arange(n, dtype=torch.float64, device="cuda")
    ua = (-U0 * torch.cos(k * x)[None, None, :] * torch.sin(k * x)[None, :, None]
          * decay).expand(n, n, n)
    peak, _ = hbm_peak()
    plane = torch.from_numpy(pkg.drivers.taylor_green_3d_populations(n, U0, Nz=1)).cuda()
    out, u64 = {}, None
    for name in ("f64", "f32", "f32dev", "f16dev", "bf16dev", "f16dev_sr", "bf16dev_sr"):
        tname, dev, bpp, label = STORAGES[name]
        dt = getattr(torch, tname)
        f = torch.empty((19, n, n, n), dtype=dt, device="cuda")
        full = _extrude(plane, n)
        if name == "f64":
            f.copy_(full)
        else:
            pkg.convert_populations(f, full, dst_deviation=dev)
        del full
        g = torch.empty_like(f)
        fd = torch.float64 if name == "f64" else torch.float32
        mom = [torch.empty((n, n, n), dtype=fd, device="cuda") for _ in range(4)]
        e0, e1 = _events()
        e0.record()
        for s in range(steps):
            m = mom if s == steps - 1 else (None,) * 4
            pkg.fused_trt_step_3d_(g, f, *m, None, n, n, n, NU, LAMBDA, periodic=(1, 1, 1),
                                   deviation=dev, stochastic_rounding=name in SR_STORAGES)
            f, g = g, f
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        u = torch.stack([t.double() for t in mom[1:]])
        del f, g, mom
        row = {"mlups": round(n ** 3 / ms / 1e3, 1),
               "hbm_frac": round(2 * 19 * bpp * n ** 3 / (ms * 1e-3) / 1e9 / peak, 4),
               "l2_vs_analytic": float(torch.linalg.vector_norm(u[0] - ua) / torch.linalg.vector_norm(ua))}
        if name == "f64":
            u64 = u
        else:
            d = u - u64
            row["l2_vs_f64"] = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(u64))
            row["max_vs_f64_over_u0"] = float(d.abs().max() / U0)
        out[name] = row
        del u
        torch.cuda.empty_cache()
    return {"workload": f"D3Q19 TRT periodic Taylor-Green {n}^3, Lambda=1/4, nu={NU}, u0={U0}, "
                        f"{steps} steps per storage", "storages": out,
            "f16dev_over_f32dev_mlups": round(out["f16dev"]["mlups"] / out["f32dev"]["mlups"], 3),
            "f16dev_sr_over_f32dev_mlups": round(out["f16dev_sr"]["mlups"] / out["f32dev"]["mlups"], 3)}


def bench_d2q9_large(pkg, n=4096, steps=50, warmup=3):
    """The 2D fused steps (fused_bgk_step!, fused_trt_step!: pull with half-way
    bounce-back on the four walls, collision, rho and u written every step as
    the reference's do) on an n x n grid larger than L2, FP64 and FP32: GLUPS
    and the fraction of the measured copy bandwidth at 2 * 9 * b bytes per
    node (the 3 * b bytes of moments count as overhead)."""
    import torch
    peak, _ = hbm_peak()
    w = torch.tensor([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=torch.float64, device="cuda")
    out = {}
    for name, dt, bpp in (("f64", torch.float64, 8), ("f32", torch.float32, 4)):
        a = (w[:, None, None] * (1 + 0.01 * torch.rand((9, n, n), dtype=torch.float64,
                                                        device="cuda"))).to(dt)
        b = torch.empty_like(a)
        mom = [torch.empty((n, n), dtype=dt, device="cuda") for _ in range(3)]
        for kern in ("bgk", "trt"):
            def step(x, y):
                if kern == "bgk":
                    pkg.fused_bgk_step_(y, x, *mom, None, n, n, 1.0 / (3 * 0.02 + 0.5))
                else:
                    pkg.fused_trt_step_(y, x, *mom, None, n, n, 0.02, 0.25)
            for _ in range(warmup):
                step(a, b)
                a, b = b, a
            e0, e1 = _events()
            e0.record()
            for _ in range(steps):
                step(a, b)
                a, b = b, a
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            out[f"{kern}_{name}"] = {"mlups": round(n * n / ms / 1e3, 1),
                                     "hbm_frac": round(2 * 9 * bpp * n * n / (ms * 1e-3) / 1e9 / peak, 4)}
        del a, b, mom
        torch.cuda.empty_cache()
    return {"workload": f"D2Q9 fused steps on a walled {n}x{n} grid, {steps} steps each", "runs": out}


def bench_unfused_paths(pkg, n2=4096, n3=256, steps=40, warmup=3):
    """Throughput of the reference's other step structures: the in-place A-A
    pair (aa_even_step!/aa_odd_step!, race-free form) and the unfused D2Q9
    cavity step (stream_2d!, apply_zou_he_north_2d!, collide_2d!) on an
    n2 x n2 walled grid, and the unfused D3Q19 walled cavity step
    (stream_3d!, Zou-He lid, collide_3d!: three launches, run_cavity_3d) at
    n3^3.  GLUPS, and the
    fraction of the measured copy bandwidth at the step's own traffic (A-A:
    2 * 9 * b per node in one buffer; unfused steps: 4 * Q * b per node, the
    stream and the collide passes each read and write every population)."""
    import torch
    peak, _ = hbm_peak()
    out = {}
    w9 = torch.tensor([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=torch.float64, device="cuda")
    w19 = torch.tensor([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=torch.float64, device="cuda")
    om = 1.0 / (3 * 0.02 + 0.5)

    def timed(step):
        for _ in range(warmup):
            step()
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    for name, dt, bpp in (("f64", torch.float64, 8), ("f32", torch.float32, 4)):
        f = (w9[:, None, None] * torch.ones((9, n2, n2), dtype=torch.float64, device="cuda")).to(dt)
        ms = timed(lambda: (pkg.aa_stream_step_2d_(f, None, None, None, None, n2, n2, om),
                            pkg.aa_local_step_2d_(f, None, None, None, None, n2, n2, om))) / 2
        out[f"aa_2d_{name}"] = {"mlups": round(n2 * n2 / ms / 1e3, 1),
                                "hbm_frac": round(2 * 9 * bpp * n2 * n2 / (ms * 1e-3) / 1e9 / peak, 4)}
        g = torch.empty_like(f)
        b2 = [f, g]

        def step2():
            pkg.stream_2d_(b2[1], b2[0], n2, n2)
            pkg.apply_zou_he_north_2d_(b2[1], 0.1, n2, n2)
            pkg.collide_2d_(b2[1], None, om)
            b2.reverse()
        ms = timed(step2)
        out[f"cavity2d_unfused_{name}"] = {
            "mlups": round(n2 * n2 / ms / 1e3, 1),
            "hbm_frac": round(4 * 9 * bpp * n2 * n2 / (ms * 1e-3) / 1e9 / peak, 4)}
        del f, g, b2
        a = (w19[:, None, None, None] * torch.ones((19, n3, n3, n3), dtype=torch.float64,
                                                   device="cuda")).to(dt)
        b = torch.empty_like(a)
        bufs = [a, b]

        def step3():
            pkg.stream_3d_(bufs[1], bufs[0], n3, n3, n3)
            pkg.apply_zou_he_top_3d_(bufs[1], 0.1, n3, n3, n3)
            pkg.collide_3d_(bufs[1], None, om)
            bufs.reverse()
        ms = timed(step3)
        out[f"cavity3d_unfused_{name}"] = {
            "mlups": round(n3 ** 3 / ms / 1e3, 1),
            "hbm_frac": round(4 * 19 * bpp * n3 ** 3 / (ms * 1e-3) / 1e9 / peak, 4)}
        del a, b, bufs
        torch.cuda.empty_cache()
    return {"workload": f"A-A pair and unfused D2Q9 cavity step on a walled {n2}^2 grid; unfused "
                        f"D3Q19 cavity step at {n3}^3; {steps} steps each", "runs": out}


def bench_thermal_guo_paths(pkg, nx2=4096, ny2=2048, n3=192, steps=20, warmup=3):
    """Throughput of the reference's unfused multi-launch steps: the
    Rayleigh-Benard DDF step (run_rayleigh_benard_2d: stream f and g, fixed
    temperature faces, T, moments, thermal BGK, Boussinesq BGK) on an
    nx2 x ny2 grid, the 3D natural-convection step (run_natural_convection_3d,
    D3Q19 f and g) at n3^3, and the Guo-forced Poiseuille steps (stream with
    x(/z) wrap and y walls, Guo BGK, force-corrected moments) in 2D and 3D.
    GLUPS and the fraction of the measured copy bandwidth at each step's own
    traffic: every launch reads its inputs and writes its outputs once,
    b bytes per value and one mask byte per node (the per-step sums are in
    the `bytes_per_node` fields)."""
    import torch
    peak, _ = hbm_peak()
    out = {}
    w9 = torch.tensor([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=torch.float64, device="cuda")
    w19 = torch.tensor([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=torch.float64, device="cuda")
    om, omT, bg = 1.0 / (3 * 0.02 + 0.5), 1.0 / (3 * 0.03 + 0.5), 1e-4

    def timed(step):
        for _ in range(warmup):
            step()
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def record(key, nodes, ms, bpn):
        out[key] = {"mlups": round(nodes / ms / 1e3, 1), "ms_per_step": round(ms, 4),
                    "bytes_per_node": bpn,
                    "hbm_frac": round(bpn * nodes / (ms * 1e-3) / 1e9 / peak, 4)}

    for name, dt, b in (("f64", torch.float64, 8), ("f32", torch.float32, 4)):
        Nx, Ny = nx2, ny2
        sh = (9, Ny, Nx)
        f = [(w9[:, None, None] * torch.ones(sh, dtype=torch.float64, device="cuda")).to(dt)
             for _ in range(2)]
        g = [(0.5 * w9[:, None, None] * torch.ones(sh, dtype=torch.float64, device="cuda")).to(dt)
             for _ in range(2)]
        T, rho, ux, uy = (torch.zeros((Ny, Nx), dtype=dt, device="cuda") for _ in range(4))
        solid = torch.zeros((Ny, Nx), dtype=torch.bool, device="cuda")

        def rb():
            pkg.stream_periodic_x_wall_y_2d_(f[1], f[0], Nx, Ny)
            pkg.stream_periodic_x_wall_y_2d_(g[1], g[0], Nx, Ny)
            pkg.apply_fixed_temp_south_2d_(g[1], 1.0, Nx)
            pkg.apply_fixed_temp_north_2d_(g[1], 0.0, Nx, Ny)
            pkg.compute_temperature_2d_(T, g[1])
            pkg.compute_macroscopic_2d_(rho, ux, uy, f[1])
            pkg.collide_thermal_2d_(g[1], ux, uy, omT)
            pkg.collide_boussinesq_2d_(f[1], T, solid, om, bg, 0.5)
            f.reverse(); g.reverse()
        # stream f, g 2*18b; T 10b; moments 12b; thermal BGK 20b; Boussinesq 19b + mask
        record(f"rayleigh_benard_2d_{name}", Nx * Ny, timed(rb), 97 * b + 1)

        def poiseuille2d():
            pkg.stream_periodic_x_wall_y_2d_(f[1], f[0], Nx, Ny)
            pkg.collide_guo_2d_(f[1], solid, om, 1e-6, 0.0)
            pkg.compute_macroscopic_2d_(rho, ux, uy, f[1])
            f.reverse()
        # stream 18b; Guo BGK 18b + mask; moments 12b
        record(f"poiseuille_guo_2d_{name}", Nx * Ny, timed(poiseuille2d), 48 * b + 1)
        del f, g, T, rho, ux, uy, solid
        torch.cuda.empty_cache()

        N = n3
        sh = (19, N, N, N)
        f = [(w19[:, None, None, None] * torch.ones(sh, dtype=torch.float64, device="cuda")).to(dt)
             for _ in range(2)]
        g = [(0.5 * w19[:, None, None, None] * torch.ones(sh, dtype=torch.float64,
                                                          device="cuda")).to(dt)
             for _ in range(2)]
        T, rho, ux, uy, uz = (torch.zeros((N, N, N), dtype=dt, device="cuda") for _ in range(5))
        solid = torch.zeros((N, N, N), dtype=torch.bool, device="cuda")

        def nc3():
            pkg.stream_3d_(f[1], f[0], N, N, N)
            pkg.stream_3d_(g[1], g[0], N, N, N)
            pkg.apply_fixed_temp_west_3d_(g[1], 1.0, N, N)
            pkg.apply_fixed_temp_east_3d_(g[1], 0.0, N, N, N)
            pkg.compute_temperature_3d_(T, g[1])
            pkg.compute_macroscopic_3d_(rho, ux, uy, uz, f[1])
            pkg.collide_thermal_3d_(g[1], ux, uy, uz, omT)
            pkg.collide_boussinesq_3d_(f[1], T, solid, om, bg, 0.5)
            f.reverse(); g.reverse()
        # stream f, g 2*38b; T 20b; moments 23b; thermal BGK 41b; Boussinesq 39b + mask
        record(f"natural_convection_3d_{name}", N ** 3, timed(nc3), 199 * b + 1)

        def poiseuille3d():
            pkg.stream_periodic_xz_wall_y_3d_(f[1], f[0], N, N, N)
            pkg.collide_guo_3d_(f[1], solid, om, 1e-6, 0.0, 0.0)
            pkg.compute_macroscopic_forced_3d_(rho, ux, uy, uz, f[1], 1e-6, 0.0, 0.0)
            f.reverse()
        # stream 38b; Guo BGK 38b + mask; forced moments 23b
        record(f"poiseuille_guo_3d_{name}", N ** 3, timed(poiseuille3d), 99 * b + 1)
        del f, g, T, rho, ux, uy, uz, solid
        torch.cuda.empty_cache()
    return {"workload": f"unfused thermal DDF and Guo-forced steps: D2Q9 {nx2}x{ny2}, D3Q19 "
                        f"{n3}^3; {steps} steps each", "runs": out}


def bench_cavity2d(pkg, steps=20000, graph_steps=200):
    """Plain FP64 D2Q9 BGK cavity 128^2, nu=0.02, u_lid=0.1 (Re=640), half-way
    bounce-back walls and moving-wall lid, from rest; `steps` fused steps
    replayed from a captured CUDA graph of `graph_steps` steps."""
    import torch
    N, nu, u = 128, 0.02, 0.1
    cfg = pkg.LBMConfig.d2q9(N, N, nu, u, 0)
    st = pkg.initialize_2d(cfg)
    w = pkg.omega(cfg)
    g = pkg.Graph()
    with g:
        a, b = st["f_in"], st["f_out"]
        for _ in range(graph_steps):
            pkg.cavity_movingwall_step_2d_(b, a, st["rho"], st["ux"], st["uy"], None, N, N, w, u)
            a, b = b, a
    g.launch()
    torch.cuda.synchronize()
    st2 = pkg.initialize_2d(cfg)
    st["f_in"].copy_(st2["f_in"])
    st["f_out"].copy_(st2["f_out"])
    e0, e1 = _events()
    e0.record()
    for _ in range(steps // graph_steps):
        g.launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ux = st["ux"].cpu().numpy()
    g.close()
    return {"workload": "D2Q9 BGK cavity 128^2 FP64, nu=0.02, u_lid=0.1, moving-wall lid, "
                        f"{steps} steps (CUDA graph of {graph_steps} fused steps)",
            "mlups": round(N * N * steps / (ms * 1e-3) / 1e6, 1), "ms": round(ms, 2),
            "max_ux_over_ulid": round(float(abs(ux).max() / u), 4),
            "finite": bool((ux == ux).all())}


def bench_batch(pkg, n_cases=256, max_steps=50000, check_every=100, tol=1e-6, storage="f16",
                autotune=True, rank=0, world=1, error_cases=0, graph=True):
    """Batched sweep: n_cases D2Q9 MRT cavities, N uniform on {64,...,512}, Re
    log-uniform [100, 2000], u_lid=0.1, one persistent launch per rank (the
    cases are split across ranks with no data exchange), replayed from a
    captured CUDA graph (graph=True).  autotune: the schedule is tuned first,
    and the tuned and the untuned (fixed) schedules' throughputs are
    reported.  With error_cases > 0, that many cases (spread over the size
    range) are rerun on the FP64 reference-arithmetic MRT cavity step for the
    same number of steps and their velocity error is reported; every case that
    went non-finite is rerun there too, to tell whether the physics or the
    storage diverges."""
    import numpy as np
    import torch
    N, nu, u, Re = pkg.sweep_cases(n_cases, seed=0)
    mine = pkg.sharding.shard_cases(N, world, rank)
    b = pkg.CavityBatch(N[mine], nu[mine], u[mine], storage)
    tune = b.autotune(trial_steps=200) if autotune else None
    g = b.capture(max_steps=max_steps, check_every=check_every, tol=tol) if graph else None
    b.reset()
    if world > 1:
        barrier(world)
    e0, e1 = _events()
    e0.record()
    if g is not None:
        g.launch()
    else:
        b.run(max_steps=max_steps, check_every=check_every, tol=tol)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    if g is not None:
        g.close()
    st = b.status()
    updates = st["updates"]
    if world > 1:
        t = torch.tensor([float(updates)], dtype=torch.float64, device="cuda")
        import torch.distributed as dist
        dist.all_reduce(t)
        updates = int(t.item())
    states, steps = {}, []
    for c in range(len(mine)):
        r = b.case(c, fields=False)
        states[r["state"]] = states.get(r["state"], 0) + 1
        steps.append(r["steps"])
    out = {"workload": f"{n_cases} D2Q9 MRT cavities, N in 64..512 step 32, Re log-uniform "
                       f"[100,2000], u_lid=0.1, {storage} deviation storage, residual {tol} or "
                       f"{max_steps} steps, one persistent cooperative launch per GPU",
           "mlups": round(updates / (ms * 1e-3) / 1e6, 1), "ms": round(ms, 1),
           "hbm_frac_36B": round(updates * 36 / (ms * 1e-3) / 1e9 / hbm_peak()[0], 4)
           if storage in ("f16", "bf16", "f16sr", "bf16sr") else None,
           "launch": "one cooperative kernel replayed from a captured CUDA graph" if graph
           else "one cooperative kernel",
           "node_updates": updates, "cases_on_rank0": states, "timed_out": st["timed_out"],
           "steps_min_median_max": [int(min(steps)), int(np.median(steps)), int(max(steps))]}
    if tune:
        tune["tuned_over_fixed"] = round(tune["best_mlups"] / tune["fixed_mlups"], 3)
        tune["fixed_schedule"] = "256-node tiles, blocks per SM at the occupancy limit (untuned default)"
        out["autotune"] = tune
    if rank == 0:
        nonfinite = []
        for c in range(len(mine)):
            r = b.case(c, fields=False)
            if r["state"] != "non-finite":
                continue
            n = int(r["N"])
            horizon = max(20000, (r["steps"] + 199) // 200 * 200)
            ux64, uy64 = _fp64_mrt_cavity(pkg, n, float(nu[mine][c]), float(u[mine][c]), horizon)
            nonfinite.append({"N": n, "Re": round(float(Re[mine][c]), 1),
                              "tau": round(3.0 * float(nu[mine][c]) + 0.5, 4),
                              "steps_in_batch": r["steps"], "fp64_steps": horizon,
                              "fp64_single_case_finite": bool(np.isfinite(ux64).all() and
                                                             np.isfinite(uy64).all())})
        out["non_finite_cases_on_fp64_path"] = nonfinite
    if error_cases and rank == 0:
        errs = []
        pick = np.unique(np.linspace(0, len(mine) - 1, error_cases).round().astype(int))
        for c in pick:
            r = b.case(int(c))
            n = int(r["N"])
            ux64, uy64 = _fp64_mrt_cavity(pkg, n, float(nu[mine][c]), float(u[mine][c]), r["steps"])
            d = np.sqrt((r["ux"] - ux64) ** 2 + (r["uy"] - uy64) ** 2)
            errs.append({"N": n, "Re": round(float(Re[mine][c]), 1), "steps": r["steps"],
                         "state": r["state"], "residual": r["residual"],
                         "max_err_over_ulid": float(np.nanmax(d) / u[mine][c]),
                         "l2_rel": float(np.sqrt(np.nansum(d ** 2) /
                                                 np.sum(ux64 ** 2 + uy64 ** 2)))})
        out["per_case_error_vs_fp64"] = errs
    b.close()
    return out


def _fp64_mrt_cavity(pkg, N, nu, u_lid, steps, graph_steps=200):
    assert graph_steps % 2 == 0
    """The plain FP64 single-case path: the fused MRT cavity step with the
    reference arithmetic (kb_cavity_mrt_step_2d), `steps` steps from rest."""
    import torch
    cfg = pkg.LBMConfig.d2q9(N, N, nu, u_lid, 0)
    st = pkg.initialize_2d(cfg)
    a, b = st["f_in"], st["f_out"]
    full, rest = divmod(steps, graph_steps)
    if full:
        g = pkg.Graph()
        with g:
            x, y = a, b
            for _ in range(graph_steps):
                pkg.cavity_mrt_step_2d_(y, x, None, None, None, None, N, N, nu, u_lid)
                x, y = y, x
        for _ in range(full):
            g.launch()          # an even number of steps: the state is back in `a`
        g.close()
    for _ in range(rest):
        pkg.cavity_mrt_step_2d_(b, a, None, None, None, None, N, N, nu, u_lid)
        a, b = b, a
    pkg.compute_macroscopic_2d_(st["rho"], st["ux"], st["uy"], a)
    torch.cuda.synchronize()
    return st["ux"].cpu().numpy(), st["uy"].cpu().numpy()


NATCONV_STORAGES = {
    # name: (torch dtype name, deviation, stochastic rounding, bytes per population)
    "f64": ("float64", False, False, 8), "f32": ("float32", False, False, 4),
    "f32dev": ("float32", True, False, 4), "f16dev_sr": ("float16", True, True, 2),
    "bf16dev_sr": ("bfloat16", True, True, 2),
}


def bench_natconv(pkg, N=512, Ra=1e5, steps=2000, FT=None, graph_steps=500, nu_ref=None,
                  storage=None):
    """Thermal DDF natural convection, N^2, Pr=0.71, fused step, `steps` steps
    replayed from a CUDA graph; returns MLUPS, the hot-wall Nusselt number
    and the final fields.  storage: f64 / f32 (the reference's arithmetic,
    f and g stored whole) or f32dev / f16dev_sr / bf16dev_sr (f - w_q and
    g - w_q T_ref, FP32 step; stochastic rounding for the 16-bit ones)."""
    import numpy as np
    import torch
    if storage is None:
        storage = "f64" if FT == torch.float64 else "f32"
    tname, dev, sr, bpp = NATCONV_STORAGES[storage]
    FT = getattr(torch, tname)
    fd = torch.float64 if storage == "f64" else torch.float32
    p = pkg.drivers.natconv_parameters(N, Ra, 0.71)
    f0 = torch.from_numpy(np.stack([pkg.lattice.D2Q9_W[q] * np.ones((N, N)) for q in range(9)]))
    g0 = torch.from_numpy(pkg.drivers.natconv_initial_g(N))

    def load(fi, fo, gi, go):
        if dev:
            pkg.convert_populations(fi, f0.cuda(), dst_deviation=True)
            gi.copy_(pkg.thermal_deviation(g0.cuda(), p["T_ref"]).to(FT))
        else:
            fi.copy_(f0.to(FT)); gi.copy_(g0.to(FT))
        fo.copy_(fi); go.copy_(gi)

    fi = torch.empty((9, N, N), dtype=FT, device="cuda")
    fo, gi, go = torch.empty_like(fi), torch.empty_like(fi), torch.empty_like(fi)
    load(fi, fo, gi, go)
    Temp = torch.zeros((N, N), dtype=fd, device="cuda")
    assert graph_steps % 2 == 0 and steps % graph_steps == 0

    def step(b, a, d, c):
        pkg.fused_natconv_step_(b, a, d, c, Temp, N, N, p["omega_f"], p["omega_T"], p["beta_g"],
                                p["T_ref"], 1.0, 0.0, deviation=dev, stochastic_rounding=sr)

    g = pkg.Graph()
    with g:
        a, b, c, d = fi, fo, gi, go
        for _ in range(graph_steps):
            step(b, a, d, c)
            a, b = b, a
            c, d = d, c
    g.launch()                      # warm-up replay (then restart from the initial state)
    torch.cuda.synchronize()
    load(fi, fo, gi, go)
    e0, e1 = _events()
    e0.record()
    for _ in range(steps // graph_steps):
        g.launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    g.close()
    T_prev = Temp.clone()
    step(fo, fi, go, gi)
    dT = float((Temp - T_prev).abs().max())
    # final fields of the populations in fi / gi (moments without the Guo
    # half-force term, as compute_macroscopic_2d!)
    fb = torch.empty((9, N, N), dtype=torch.float64, device="cuda")
    if dev:
        pkg.convert_populations(fb, fi, src_deviation=True)
        gb = pkg.thermal_deviation(gi, p["T_ref"], to_deviation=False)
    else:
        fb.copy_(fi); gb = gi.double()
    rho = fb.sum(0)
    ux = (fb[1] - fb[3] + fb[5] - fb[6] - fb[7] + fb[8]) / rho
    uy = (fb[2] - fb[4] + fb[5] + fb[6] - fb[7] - fb[8]) / rho
    T = gb.sum(0).cpu().numpy()
    out = {"workload": f"thermal DDF natural convection {N}^2 {storage}, Ra={Ra:g}, "
                       f"Pr=0.71, {steps} fused steps (CUDA graph of {graph_steps})",
           "mlups": round(N * N * steps / (ms * 1e-3) / 1e6, 1),
           "gbs_alg": round(N * N * steps * 36 * bpp / (ms * 1e-3) / 1e9, 1),
           "Nu": pkg.drivers.nusselt_hot_wall(T), "max_dT_last_step": dT}
    if nu_ref is not None:
        out["Nu_de_vahl_davis"] = nu_ref
    return out, T, ux.cpu().numpy(), uy.cpu().numpy()


def bench_natconv_validation(pkg, N=512, steps_by_ra=None,
                             storages=("f32", "f32dev", "f16dev_sr")):
    """Config 4: Nu, MLUPS and the errors of T and u against the FP64 run for
    Ra in {1e4, 1e5, 1e6} on N^2, per storage: FP32 with f and g whole (the
    reference's arithmetic), FP32 deviations, FP16 deviations with
    stochastic rounding."""
    import json as _json
    import numpy as np
    pins = _json.loads((ROOT / "tests" / "golden" / "reference_pins.json").read_text())
    dvd = pins["de_vahl_davis_nu"]
    steps_by_ra = steps_by_ra or {1e4: 1280000, 1e5: 2560000, 1e6: 2560000}
    res = {}
    for ra, steps in steps_by_ra.items():
        r64, T64, ux64, uy64 = bench_natconv(pkg, N, ra, steps, storage="f64",
                                             nu_ref=dvd.get(str(int(ra))))
        un = np.sqrt(np.sum(ux64 ** 2 + uy64 ** 2))
        row = {"fp64": r64}
        for st in storages:
            r, T, ux, uy = bench_natconv(pkg, N, ra, steps, storage=st)
            r["T_max_err_vs_fp64"] = float(np.max(np.abs(T - T64)))
            r["u_l2_rel_vs_fp64"] = float(np.sqrt(np.sum((ux - ux64) ** 2 + (uy - uy64) ** 2)) / un)
            r["Nu_rel_err_vs_fp64"] = float(abs(r["Nu"] - r64["Nu"]) / r64["Nu"])
            row[st] = r
        res[f"Ra={ra:g}"] = row
    return res


def bench_warmstart(pkg, N=256, n_train=2000, n_test=64, epochs=40, batch=16, base=32,
                    data_steps=200000, data_tol=1e-6, tol=1e-8, max_steps=2000000,
                    check_every=1000, init_iters=500, grad_weight=200.0, seed=0):
    """Learned warm start: train the encoder-decoder on the steady N^2 cavities
    among n_train run by the batched kernel (Re log-uniform [100, 3200], u_lid
    0.1) to r_u <= data_tol within data_steps: only the cases that reached it
    are training targets (an unconverged field is a transient, not a steady
    solution; FP32 storage puts a floor near 1e-7 under r_u, so data_tol is
    1e-6),
    then run n_test held-out cases to r_u <= tol with the plain FP64 MRT step
    from rest (cold), from the network's prediction (warm) and, as the bound
    of the method, from the cold run's own converged field (ideal).  Warm and
    ideal starts run init_iters consistent-initialisation iterations first
    (counted as steps).  Reports data, training and inference throughput,
    steps and wall time to steady, and the converged-field differences."""
    import numpy as np
    import torch
    from importlib import import_module
    sur = import_module(pkg.__name__ + ".surrogate")
    out = {"workload": f"learned warm start, {N}^2 lid-driven MRT cavities, Re log-uniform "
                       f"[100,3200], u_lid=0.1; {n_train} training / {n_test} held-out cases; "
                       f"4-level U-Net, {base} base channels, BF16 tcgen05, batch {batch}, "
                       f"{epochs} epochs, loss MSE + {grad_weight:g} x gradient term; plain FP64 "
                       f"MRT to r_u <= {tol:g} (cap {max_steps} steps)"}
    re_tr, re_te = sur.held_out_split(n_train, n_test, seed=seed)
    e0, e1 = _events()
    e0.record()
    fields, info = sur.steady_cavities(re_tr, N, storage="f32", max_steps=data_steps,
                                       tol=data_tol, check_every=500)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    steps = np.array([s for s, _, _ in info])
    states = [st for _, _, st in info]
    out["data"] = {"storage": "f32 f-w, FP32 MRT, batched persistent kernel", "ms": round(ms, 1),
                   "mlups": round(float(steps.sum()) * N * N / (ms * 1e-3) / 1e6, 1),
                   "steps_min_median_max": [int(steps.min()), int(np.median(steps)), int(steps.max())],
                   "states": {k: states.count(k) for k in set(states)}}
    ok = torch.tensor([st == "converged" for st in states])
    keep = torch.nonzero(ok).flatten()
    out["data"]["training_targets"] = int(ok.sum())
    fields = fields.index_select(0, keep.cuda())
    re_tr = re_tr[keep.numpy()]
    model = sur.Surrogate(max_batch=batch, H=N, W=N, base_channels=base, seed=seed)
    e0.record()
    hist = sur.train(model, re_tr, fields, epochs=epochs, batch=batch, lr=1e-3, lr_min=2e-5,
                     grad_weight=grad_weight)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    nsteps = epochs * (len(re_tr) // batch)
    _, tfl = model.flops(batch)
    out["train"] = {"params": model.n_params, "steps": nsteps, "ms": round(ms, 1),
                    "tflops": round(tfl * nsteps / (ms * 1e-3) / 1e12, 1),
                    "loss_first_last": [hist[0], hist[-1]], "timed_out": model.timed_out()}
    del fields
    torch.cuda.synchronize()
    e0.record()
    preds = []
    for i in range(0, n_test, batch):
        x = model.inputs(re_te[i:i + batch], n_nodes=N)
        preds.append(model.infer(x))
    pred = torch.cat(preds)
    e1.record()
    torch.cuda.synchronize()
    infer_ms = e0.elapsed_time(e1)
    ffl, _ = model.flops(batch)
    out["inference"] = {"ms": round(infer_ms, 2),
                        "tflops": round(ffl * (n_test / batch) / (infer_ms * 1e-3) / 1e12, 1)}
    cold = [sur.PlainCavity(N, 0.1 * N / r, 0.1, check_every=check_every) for r in re_te]
    t_cold = sur.run_to_steady(cold, tol=tol, max_steps=max_steps, check_every=check_every)
    exact = torch.stack([c.fields() for c in cold])
    runs = {}
    for name, init in (("warm", pred), ("ideal", exact)):
        cs = [sur.PlainCavity(N, 0.1 * N / r, 0.1, check_every=check_every, init=init[c],
                              init_iters=init_iters) for c, r in enumerate(re_te)]
        t = sur.run_to_steady(cs, tol=tol, max_steps=max_steps, check_every=check_every)
        runs[name] = (cs, t)
    sc = np.array([c.steps for c in cold])
    conv_c = np.array([c.residual <= tol for c in cold])
    res = {"inference_ms": round(infer_ms, 2), "cold_wall_s": round(t_cold, 2),
           "cold_converged": int(conv_c.sum()), "re": [round(float(r), 1) for r in re_te],
           "cold_steps": sc.tolist()}
    for name, (cs, t) in runs.items():
        sw = np.array([c.steps for c in cs])
        conv = np.array([c.residual <= tol for c in cs])
        both = conv & conv_c
        dmax = [float((c.fields()[1:] - w.fields()[1:]).abs().max()) / 0.1
                for c, w, b in zip(cold, cs, both) if b]
        per_threshold = {}
        for th in sur.THRESHOLDS:
            pairs = [(c.reached[th], w.reached[th]) for c, w in zip(cold, cs)
                     if th in c.reached and th in w.reached]
            if pairs:
                a = sum(p[0] for p in pairs)
                b = sum(p[1] for p in pairs)
                per_threshold[f"{th:g}"] = {"cases": len(pairs), "cold_steps": a, "steps": b,
                                            "ratio": round(a / max(1, b), 3)}
        res[name] = {"steps": sw.tolist(), "converged": int(conv.sum()),
                     "wall_s": round(t + (infer_ms * 1e-3 if name == "warm" else 0.0), 2),
                     "steps_ratio_cold_over_this_on_cases_both_converged":
                         round(float(sc[both].sum()) / max(1.0, float(sw[both].sum())), 3),
                     "per_residual_threshold": per_threshold,
                     "converged_max_du_over_ulid": max(dmax) if dmax else None}
        for c in cs:
            c.close()
    res["prediction_l2_rel_u_vs_cold_field"] = [
        float((pred[k, 1:].double() - exact[k, 1:]).norm() / exact[k, 1:].norm())
        for k in range(n_test)]
    for c in cold:
        c.close()
    out["held_out"] = res
    model.close()
    return out


def bench_surrogate(pkg, steps=10, warmup=3, batch=16, N=256, base=32, engine=None):
    """Throughput of the warm-start network on the tensor cores: `steps` timed
    training steps (forward, MSE + gradient-term loss, backward, Adam) and
    forward passes of `batch` cavities at N^2, after `warmup` untimed steps;
    TFLOP/s against the measured dense BF16 peak."""
    import numpy as np
    import torch
    from importlib import import_module
    sur = import_module(pkg.__name__ + ".surrogate")
    if engine is not None:
        pkg.set_umma_engine(engine)
    m = sur.Surrogate(max_batch=batch, H=N, W=N, base_channels=base, seed=0)
    m.set_grad_weight(200.0)
    re = np.exp(np.random.default_rng(0).uniform(np.log(100.0), np.log(3200.0), batch))
    x = m.inputs(re, N)
    tgt = torch.zeros((batch, 3, N, N), device="cuda")
    tgt[:, 0] = 1.0
    fwd, trn = m.flops(batch)
    for _ in range(warmup):
        m.train_step(x, tgt, 1e-5)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        m.train_step(x, tgt, 1e-5)
    e1.record()
    torch.cuda.synchronize()
    ms_t = e0.elapsed_time(e1) / steps
    e0.record()
    for _ in range(steps):
        m.infer(x)
    e1.record()
    torch.cuda.synchronize()
    ms_i = e0.elapsed_time(e1) / steps
    peak = None
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            peak = d.get("bf16_tflops_sustained") or d.get("bf16_tflops")
        except (ValueError, OSError):
            peak = None
    peak = float(peak) if peak else 1390.0
    out = {"workload": f"warm-start U-Net, {N}^2, batch {batch}, {base} base channels, BF16 "
                       f"tcgen05, engine {2 if engine is None else engine}",
           "train_ms": round(ms_t, 3), "train_tflops": round(trn / (ms_t * 1e-3) / 1e12, 1),
           "infer_ms": round(ms_i, 3), "infer_tflops": round(fwd / (ms_i * 1e-3) / 1e12, 1),
           "bf16_peak_tflops": peak,
           "train_frac_of_peak": round(trn / (ms_t * 1e-3) / 1e12 / peak, 4),
           "timed_out": m.timed_out()}
    m.close()
    if engine is not None:
        pkg.set_umma_engine(2)
    return out


def bench_libb(pkg, N=256, R=40.0, steps=50, warmup=5):
    """TRT + interpolated bounce-back around a sphere of radius R at the
    centre of a periodic N^3 box (moving fluid, stationary wall): MLUPS of the
    reference-layout step (dense per-link arrays) and of the compact cut-link
    table, per storage, against the HBM roofline of 2*19*b bytes per node."""
    import torch
    peak, _ = hbm_peak()
    c = (N - 1) / 2.0
    qw64, solid = pkg.libb.precompute_q_wall_sphere_3d_torch(N, N, N, c, c, c, R, device="cuda")
    m = solid.to(torch.uint8)
    n_links = int((qw64 > 0).sum().item())
    nodes = N ** 3
    W = torch.tensor([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=torch.float64, device="cuda")
    out = {"workload": f"D3Q19 TRT + LI-BB, sphere R={R} in a periodic {N}^3 box, nu=0.01, "
                       f"Lambda=3/16, {steps} steps", "solid_nodes": int(solid.sum().item()),
           "cut_links": n_links, "peak_gbs": peak, "runs": {}}

    def timeit(step, fa, fb):
        for _ in range(warmup):
            step(fa, fb)
            fa, fb = fb, fa
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            step(fa, fb)
            fa, fb = fb, fa
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def record(name, ms, b):
        gbs = 2 * 19 * b * nodes / (ms * 1e-3) / 1e9
        out["runs"][name] = {"ms": round(ms, 4), "mlups": round(nodes / ms / 1e3, 1),
                             "gbs": round(gbs, 1), "hbm_frac": round(gbs / peak, 4)}

    per = (True, True, True)
    for dt, b in ((torch.float64, 8), (torch.float32, 4)):
        qw = qw64.to(dt)
        zeros = torch.zeros_like(qw)
        f0 = (W.view(19, 1, 1, 1) * torch.ones((19, N, N, N), dtype=torch.float64, device="cuda")).to(dt)
        fa, fb = f0.clone(), torch.empty_like(f0)
        name = "f64" if dt == torch.float64 else "f32"
        ms = timeit(lambda x, y: pkg.fused_trt_libb_v2_step_3d_(
            y, x, None, None, None, None, m, qw, zeros, zeros, zeros, N, N, N, 0.01,
            periodic=per), fa, fb)
        record(f"{name}_dense", ms, b)
        links = pkg.libb.CutLinks(m, qw, zeros, zeros, zeros)
        ms = timeit(lambda x, y: pkg.fused_trt_libb_links_step_3d_(
            y, x, None, None, None, None, links, 0.01, periodic=per), fa, fb)
        record(f"{name}_table", ms, b)
        ms = timeit(lambda x, y: pkg.fused_trt_step_3d_(
            y, x, None, None, None, None, m, N, N, N, 0.01, 3 / 16, periodic=per), fa, fb)
        record(f"{name}_no_links", ms, b)
        if dt == torch.float32:
            for sname, sdt, sb in (("f32dev", torch.float32, 4), ("f16dev", torch.float16, 2),
                                   ("bf16dev", torch.bfloat16, 2)):
                ga = torch.zeros((19, N, N, N), dtype=sdt, device="cuda")
                gb = torch.empty_like(ga)
                ms = timeit(lambda x, y: pkg.fused_trt_libb_links_step_3d_(
                    y, x, None, None, None, None, links, 0.01, periodic=per,
                    deviation=True), ga, gb)
                record(f"{sname}_table", ms, sb)
                del ga, gb
        out["nodes_with_links"] = links.nodes_with_links()
        links.close()
        del qw, zeros, f0, fa, fb
        torch.cuda.empty_cache()
    return out


def bench_output(pkg, n=256, steps=400, every=20):
    """Cost of field output in a step loop: the periodic D3Q19 TRT Taylor-Green
    step (n^3, F32 f-w) with rho, ux, uy, uz written every `every` steps and
    copied to the host (a) not at all, (b) synchronously (the reference's
    Array() per snapshot), (c) through the asynchronous snapshot pipeline
    (staging copy, device-to-host on a copy stream, host sink on a thread).
    Wall-clock ms per step, host synchronised at both ends."""
    import time
    import torch
    plane = torch.from_numpy(pkg.drivers.taylor_green_3d_populations(n, U0, Nz=1)).cuda()
    f = torch.empty((19, n, n, n), dtype=torch.float32, device="cuda")
    full = _extrude(plane, n)
    pkg.convert_populations(f, full, dst_deviation=True)
    del full
    g = torch.empty_like(f)
    mom = [torch.empty((n, n, n), dtype=torch.float32, device="cuda") for _ in range(4)]
    got = []
    snaps = pkg.output.AsyncSnapshots(lambda s, t, fl: got.append(s), depth=3)

    def run(mode):
        nonlocal f, g
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(steps):
            out = (s + 1) % every == 0
            m = mom if out else [None] * 4
            pkg.fused_trt_step_3d_(g, f, *m, None, n, n, n, NU, 0.25, periodic=(1, 1, 1),
                                   deviation=True)
            f, g = g, f
            if out and mode == "sync":
                [t.cpu() for t in mom]
            elif out and mode == "async":
                snaps.submit(s + 1, {"rho": mom[0], "velocity": tuple(mom[1:])})
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        return (t1 - t0) * 1e3 / steps

    run("none")
    run("async")   # allocates the pinned ring once; the timed runs reuse it
    res = {m: round(run(m), 4) for m in ("none", "sync", "async", "none")}
    snaps.close()
    snap_mb = 4 * n ** 3 * 4 / 1e6
    host = torch.empty(mom[0].shape, dtype=torch.float32, pin_memory=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(10):
        host.copy_(mom[0], non_blocking=True)
    torch.cuda.synchronize()
    d2h = 10 * mom[0].numel() * 4 / (time.perf_counter() - t0) / 1e9
    return {"workload": f"D3Q19 TRT Taylor-Green {n}^3 f32dev, rho/u ({snap_mb:.0f} MB) every "
                        f"{every} of {steps} steps", "ms_per_step": res,
            "pinned_d2h_gbs": round(d2h, 1),
            "async_snapshots_delivered": len(got),
            "sync_overhead_ms_per_snapshot": round((res["sync"] - res["none"]) * every, 3),
            "async_overhead_ms_per_snapshot": round((res["async"] - res["none"]) * every, 3)}


def bench_slab(pkg, n, storage, steps, warmup, rank, world):
    """One periodic n^3 Taylor-Green grid split along z over `world` ranks
    (strong scaling): per step the fused TRT step on each slab's local array
    and the exchange of the five crossing populations per face (NCCL
    point-to-point; with one rank, copies of the slab's own end planes).
    Timed on the device with CUDA events, max over ranks."""
    import torch
    tname, deviation, bpp, _ = STORAGES[storage]
    dt = getattr(torch, tname)
    slab = pkg.slab.Slab(n, world, rank, True)
    plane = torch.from_numpy(pkg.drivers.taylor_green_3d_populations(n, U0, Nz=1)).cuda()
    a = torch.empty((19, slab.nz_alloc, n, n), dtype=dt, device="cuda")
    pkg.convert_populations(a, plane.expand(19, slab.nz_alloc, n, n).contiguous(),
                            dst_deviation=deviation)
    b = torch.empty_like(a)
    st = pkg.slab.SlabTRT3D(slab, n, n, nu=NU, Lambda=LAMBDA, periodic_xy=(1, 1),
                            deviation=deviation, stochastic_rounding=storage in SR_STORAGES)
    out = {}
    # the whole local array then the exchange (step), and the face planes,
    # the exchange posted, then the interior planes (step_overlapped)
    for key, fn in (("mlups", st.step), ("mlups_overlapped", st.step_overlapped)):
        for _ in range(warmup):
            fn(b, a)
            a, b = b, a
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            fn(b, a)
            a, b = b, a
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        out[key] = round(n ** 3 * steps / (ms * 1e-3) / 1e6, 1)
        out["ms_per_step" if key == "mlups" else "ms_per_step_overlapped"] = round(ms / steps, 4)
    halo = 2 * 5 * n * n * bpp if world > 1 else 0
    return {"workload": f"D3Q19 TRT periodic Taylor-Green {n}^3 split along z over {world} "
                        f"rank(s), {storage}", "scaling": "strong", **out,
            "planes_per_rank": slab.nz, "ghost_planes_per_rank": slab.nz_alloc - slab.nz,
            "halo_bytes_sent_per_rank_per_step": halo}


def bench_slab2d(pkg, steps, warmup, rank, world, Nx=4096, Ny=4096):
    """One walled Nx x Ny D2Q9 grid (fused TRT, FP64 and FP32) split along y
    over `world` ranks (strong scaling): per step the fused step on each
    slab's local rows and the exchange of the three crossing populations per
    face (NCCL point-to-point).  Timed on the device with CUDA events, max
    over ranks."""
    import torch
    slab = pkg.slab.Slab(Ny, world, rank, False)
    w9 = torch.tensor([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, dtype=torch.float64, device="cuda")
    out = {}
    for name, dt, b in (("f64", torch.float64, 8), ("f32", torch.float32, 4)):
        a = (w9[:, None, None] * torch.ones((9, slab.nz_alloc, Nx), dtype=torch.float64,
                                           device="cuda")).to(dt)
        c = torch.empty_like(a)
        st = pkg.slab.SlabD2Q9(slab, Nx, "trt", nu=NU, Lambda=LAMBDA)
        for _ in range(warmup):
            st.step(c, a)
            a, c = c, a
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            st.step(c, a)
            a, c = c, a
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        out[name] = {"mlups": round(Nx * Ny * steps / (ms * 1e-3) / 1e6, 1),
                     "ms_per_step": round(ms / steps, 4),
                     "halo_bytes_sent_per_rank_per_step":
                         (int(slab.lo) + int(slab.hi)) * 3 * Nx * b}
        del a, c
        torch.cuda.empty_cache()
    return {"workload": f"walled D2Q9 TRT {Nx}x{Ny} split along y over {world} rank(s)",
            "scaling": "strong", "rows_per_rank": slab.nz, "runs": out}


def _extrude(plane, n):
    import torch
    out = torch.empty((19, n, n, n), dtype=plane.dtype, device=plane.device)
    out.copy_(plane.expand(19, n, n, n))
    return out


def run_other(args):
    """One of the other configurations, printed as its own JSON line."""
    import torch
    import __graft_entry__ as graft
    rank, world, _ = dist_setup(args.gpus)
    pkg = graft.load_package()
    pkg._lib.load()
    pkg.set_trt3d_variant(args.trt_variant)
    r = None
    if args.workload == "cavity2d":
        if rank == 0:
            r = bench_cavity2d(pkg, steps=max(args.steps, 200) // 200 * 200)
    elif args.workload == "batch":
        r = bench_batch(pkg, n_cases=args.cases, max_steps=args.max_steps, rank=rank,
                        world=world, error_cases=(8 if world == 1 and args.cases == 256 else 0),
                        storage=args.batch_storage, autotune=not args.no_autotune)
    elif args.workload == "warmstart":
        if rank == 0:
            r = bench_warmstart(pkg)
    elif args.workload == "surrogate":
        if rank == 0:
            r = bench_surrogate(pkg, steps=min(args.steps, 50), warmup=args.warmup)
    elif args.workload == "output":
        if rank == 0:
            r = bench_output(pkg, n=args.grid)
    elif args.workload == "slab":
        r = bench_slab(pkg, args.grid, args.storage, max(args.steps, 20), args.warmup, rank, world)
    elif args.workload == "slab2d":
        r = bench_slab2d(pkg, max(args.steps, 20), args.warmup, rank, world)
    elif args.workload == "libb":
        if rank == 0:
            r = bench_libb(pkg, N=args.grid, R=40.0 * args.grid / 256,
                           steps=min(max(args.steps, 20), 200), warmup=args.warmup)
    elif args.workload == "thermal":
        if rank == 0:
            r = bench_thermal_guo_paths(pkg, steps=min(max(args.steps, 4), 200), warmup=args.warmup)
    elif rank == 0:
        r = bench_natconv_validation(pkg)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "workload": args.workload, "n_gpus": world,
                          "result": r}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--storage", default="f32dev", choices=sorted(STORAGES))
    ap.add_argument("--batch-storage", default="f16", choices=["f16", "bf16", "f32", "f16sr", "bf16sr"],
                    help="population storage of --workload batch (sr: stochastic rounding)")
    ap.add_argument("--trt-variant", type=int, default=0,
                    help="deviation-storage TRT kernel: 0 automatic, 1 node, 2 x/x+32 pairs, "
                         "3 vector pairs, 4 16-bit quads, 5 staged row tiles (two rows where Ny "
                         "is even), 6 staged one-row tiles")
    ap.add_argument("--grid", type=int, default=N_GRID)
    ap.add_argument("--cases", type=int, default=256, help="--workload batch: number of cavities")
    ap.add_argument("--max-steps", type=int, default=50000,
                    help="--workload batch: step cap per cavity")
    ap.add_argument("--no-autotune", action="store_true",
                    help="--workload batch: skip the schedule autotuner")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the short measurements of the other configurations")
    ap.add_argument("--workload", default="tgv3d", choices=["tgv3d", "cavity2d", "batch", "natconv", "warmstart", "surrogate", "slab", "slab2d",
                             "libb", "output", "thermal"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "tgv3d":
        return run_other(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
