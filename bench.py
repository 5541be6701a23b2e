"""Benchmark of the GeoSWE fused finite-volume step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gsw|reference] [--n 8192]

Workload (the rain-on-terrain pluvial case, dense grid): 8192 x 8192 cells, dx = 3 m,
seeded fractal bed (power ~ k^-3, 0-40 m, 0.2 % slope), 4 Manning classes
(0.025/0.04/0.06/0.1) on 256 seeded Voronoi cells, dry start, uniform rain 50 mm/h,
x+ edge open ('fall'), other edges walls, CFL 0.5, fp32. A step is one time step of the
solver (ghost fill + fused SRM-HLLC/rain/Euler/Manning/wet-dry step + device dt).
The state (3 x 268 MB) is far larger than L2, so no flush is needed between steps.

Prints one JSON line. Under torchrun each rank runs an independent replica (the
single-GPU step does not shard here), timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s on 1 B200: plain vs batched; adjoint/forward cost ratio"
UNIT = "cell-updates/s"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """SM clock and clock-event reasons sampled during a timed region. NVML is polled
    from a thread every 5 ms, with one sample at start() and one at stop(), so a region
    of a few tens of milliseconds is covered too; nvidia-smi (200 ms) is the fallback.
    Reads only: no clock or other GPU setting is changed."""
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index=0):
        self.index = index
        self.samples = []            # (sm MHz, reasons bitmask)
        self.smax = None
        self._h = None
        self._stop = threading.Event()
        self._thread = None
        self._smi = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:   # the CUDA device's own NVML handle (CUDA_VISIBLE_DEVICES may renumber)
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        import pynvml
        sm = pynvml.nvmlDeviceGetClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        self.samples.append((float(sm), int(rs)))

    def _poll(self):
        while not self._stop.wait(0.005):
            try:
                self._sample()
            except Exception:
                return

    def start(self):
        try:
            import pynvml
            self._h = self._handle()
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
            self._sample()
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
        except Exception:
            self._h = None
            self._start_smi()

    def _start_smi(self):
        q = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._smi = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._lines = []
            self._thread = threading.Thread(target=lambda: self._lines.extend(ln.strip() for ln in self._smi.stdout),
                                            daemon=True)
            self._thread.start()
        except Exception:
            self._smi = None

    def stop(self):
        if self._h is not None:
            self._stop.set()
            self._thread.join(timeout=1.0)
            try:
                self._sample()
            except Exception:
                pass
        elif self._smi is not None:
            self._smi.terminate()
            try:
                self._smi.wait(timeout=5)
            except Exception:
                self._smi.kill()
            bits = [self.REASONS[k] for k in ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                              "sw_power_cap")]
            for ln in self._lines:
                f = [x.strip() for x in ln.split(",")]
                try:
                    sm, self.smax = float(f[1]), float(f[2])
                except (ValueError, IndexError):
                    continue
                self.samples.append((sm, sum(b for b, v in zip(bits, f[3:7]) if v.lower().startswith("active"))))
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no NVML or nvidia-smi"], "samples": 0}
        sm = [s for s, _ in self.samples]
        mask = 0
        for _, r in self.samples:
            mask |= r
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                "reasons": sorted(k for k, b in self.REASONS.items() if mask & b), "samples": len(sm),
                "source": "nvml" if self._h is not None else "nvidia-smi"}


def build_case(n, dtype="float32", seed=0):
    """Host arrays of the rain-on-terrain case (the bed and classes are computed once and
    cached under _bench_cache/ as .npy, keyed by size and seed)."""
    from geoswe_b200.synthetic import fractal_bed, voronoi_classes_fast
    cache = ROOT / "_bench_cache"
    cache.mkdir(exist_ok=True)
    fz, fc = cache / f"bed_{n}_{seed}.npy", cache / f"cls_{n}_{seed}.npy"
    if fz.exists() and fc.exists():
        z, cls = np.load(fz), np.load(fc)
    else:
        z = fractal_bed(n, n, 3.0, seed=seed).astype(np.float32)
        cls = voronoi_classes_fast(n, n, seed=seed)
        np.save(fz, z)
        np.save(fc, cls)
    return z, cls


def make_solver(z, cls, n, dtype="float32", arith="exact", block=None, comm=None, dims=None, q0=None,
                clsp=None):
    """The rain-on-terrain solver; with `block` = (x0, x1, y0, y1) and `comm`, this rank's
    block of the domain split over the ranks of `comm`. `q0` and `clsp` (the padded
    classes) may be given as the caller holds them (the end-to-end measurement passes
    page-locked arrays)."""
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.synthetic import MANNING_CLASSES
    x0, x1, y0, y1 = block if block is not None else (0, n, 0, n)
    mesh = Mesh2D(nx=x1 - x0, ny=y1 - y0, dx=3.0, dy=3.0, ngh=2)
    cfg = Config(bc_x="wall", bc_y="wall", bc={"x+": "fall"}, cfl=0.5, dtype=dtype,
                 friction="manning", arith=arith,
                 rainfall_forcing=RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0]))
    if q0 is None:
        q0 = np.zeros((3, x1 - x0, y1 - y0), np.float32)
    zb = z if block is None else z[x0:x1, y0:y1]
    s = Solver2D(mesh, cfg, q0, zb, comm=comm, dims=dims)
    ngh = mesh.ngh
    if clsp is None:
        clsp = np.ascontiguousarray(np.pad(cls, ngh, mode="edge")[x0:x1 + 2 * ngh, y0:y1 + 2 * ngh])
    s.set_manning_table(clsp, MANNING_CLASSES)
    return s


def counters():
    """Per-kernel ncu counters from profiles/counters.json: DRAM bytes per updated cell
    (dram__bytes_read.sum + dram__bytes_write.sum of one launch / its cells; the traffic
    is proportional to the cells, so it scales to a launch of another size) and warp
    instructions per updated cell (smsp__inst_executed.sum / cells; with the SM clock,
    the instruction-issue roofline: one warp instruction per scheduler per cycle, four
    schedulers per SM). Each entry names the sources its kernel is compiled from and
    their hash when it was captured; `current_build` says whether those sources are the
    ones measured here."""
    p = ROOT / "profiles" / "counters.json"
    d = json.loads(p.read_text()) if p.exists() else {}
    try:
        from geoswe_b200.build import source_hash
    except Exception:
        source_hash = None
    for v in d.values():
        cur = source_hash(v.get("files")) if source_hash is not None else None
        v["current_build"] = cur is not None and v.get("sources") == cur
    return d


def _traffic(kind, cells):
    c = counters().get(kind)
    if not c or c.get("dram_bytes_per_cell") is None:
        return None, None
    return (c["dram_bytes_per_cell"] * cells / 1e9,
            {"unit": "GB per launch", "source": f"profiles/counters.json[{kind}] ({c.get('workload')})",
             "dram_bytes_per_cell": c["dram_bytes_per_cell"], "captured_on_sources": c.get("sources"),
             "current_build": c["current_build"]})


def issue_roofline(kind, cells, kern_ms, clocks):
    """Issue-rate roofline of a step kernel: achieved warp instructions per second (the
    ncu count per cell x cells / the CUDA-event launch time) against 4 x SMs x the
    sampled SM clock (max clock when no sample)."""
    import torch
    c = counters().get(kind)
    if not c or c.get("warp_inst_per_cell") is None:
        return None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    peak = 4.0 * sms * mhz * 1e6
    ipc = c["warp_inst_per_cell"]
    achieved = ipc * cells / (kern_ms / 1e3)
    return {"bound": "instruction issue", "warp_inst_per_cell": ipc,
            "achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "sm_mhz": mhz, "source": f"profiles/counters.json[{kind}] ({c.get('workload')})",
            "captured_on_sources": c.get("sources"), "current_build": c["current_build"]}


def max_over_ranks(x, device):
    """The maximum of a per-rank time over the process group (every rank gets it)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def dense_config(n, world):
    """The `config` of the default line (both arms)."""
    return {"workload": f"rain-on-terrain dense {n}x{n}, dx=3 m, fractal bed, 4-class Voronoi Manning, dry "
                        f"start, 50 mm/h uniform rain, x+ open, walls elsewhere, CFL 0.5, fp32",
            "cells": n * n, "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"}


def bytes_per_cell(track_max=True):
    # read h, hu, hv, z (16 B) + class id (1 B); write h, hu, hv (12 B); running max 8 B
    return 16 + 1 + 12 + (8 if track_max else 0)


def measure_dense(args, z, cls, n, world, arith="exact"):
    """Device-resident throughput of the dense rain-on-terrain run with one arithmetic:
    warm-up, launch-shape tuning, a warm-up of the timed window (its graph is captured
    there), then exactly `steps` timed steps between CUDA events; then the step
    kernel alone (CUDA events, same launch shape) for the roofline."""
    import torch
    s = make_solver(z, cls, n, arith=arith)
    forced = args.fast_shape if arith == "fast" else args.exact_shape
    if forced:
        s._tile_rows, s._warps, s._min_blocks = (int(v) for v in forced.split(","))
    s.run(t_end=1e12, max_steps=args.warmup)
    tune = None
    if not forced and not args.no_tune:
        from geoswe_b200 import autotune
        best, table = autotune.tune_dense(s, reps=4)
        s._tile_rows, s._warps, s._min_blocks = best["tile_rows"], best["warps"], best["min_blocks"]
        tune = {"best": best, "table": table}
    # warm-up with the timed run's window and launch shape: its CUDA graph is captured here
    s.run(t_end=1e12, max_steps=args.warmup, window=s._window_size())
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = Clocks(int(os.environ.get("LOCAL_RANK", 0)))
    clk.start()
    l0 = s.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    steps = s.run(t_end=1e12, max_steps=args.steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    launches = s.kernel_launches - l0
    assert steps == args.steps, (steps, args.steps)
    torch.cuda.nvtx.range_push("kernel_timing")        # the launches an ncu capture targets
    kern_ms = time_step_kernel(s, reps=args.kernel_reps)
    torch.cuda.nvtx.range_pop()
    shape = {"tile_rows": s._tile_rows or "auto", "warps": s._warps or 4, "min_blocks": s._min_blocks}
    del s
    torch.cuda.empty_cache()
    if world > 1:
        ms = max_over_ranks(ms, "cuda")
    return dict(ms=ms, launches=launches, kern_ms=kern_ms, clocks=clocks, shape=shape, tune=tune)


def run_gsw(args, rank, world):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    n = args.n
    z, cls = build_case(n)
    cells = n * n
    # ---------------- device-resident throughput (value), exact arithmetic ----------------
    m = measure_dense(args, z, cls, n, world, args.dense_arith)
    ms, kern_ms = m["ms"], m["kern_ms"]
    # ---------------- end to end through the public API ----------------
    e2e = run_e2e(args, z, cls, n, world)
    torch.cuda.empty_cache()
    value = cells * args.steps * world / (ms / 1e3)
    peak, peak_kind = _peaks()
    bpc = bytes_per_cell(True)
    achieved = bpc * cells / (kern_ms / 1e3) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dense_config(n, world),
        "e2e": e2e,
        "gpu_launches": int(m["launches"]),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": _traffic("dense", cells)[0],
                     "traffic_from": _traffic("dense", cells)[1],
                     "kernel": "dense_march_kernel<float,true>", "kernel_ms": kern_ms,
                     "bytes_per_cell": bpc, "peak_source": peak_kind},
        "issue": issue_roofline("dense", cells, kern_ms, m["clocks"]),
        "clocks": m["clocks"],
        "arith": ("exact (IEEE, powf Manning power: bit-identical to the reference kernel without FMA contraction)"
                  if args.dense_arith == "exact" else "portable (IEEE, Newton Manning power)"),
        "launch_shape": m["shape"],
    }
    if m["tune"] is not None:
        out["autotune"] = m["tune"]
    # ---------------- the opt-in fast arithmetic, same workload ----------------
    if not args.no_fast:
        f = measure_dense(args, z, cls, n, world, "fast")
        f_ach = bpc * cells / (f["kern_ms"] / 1e3) / 1e9
        out["fast_arith"] = {
            "what": "Config(arith='fast'): FMA contraction, approximate binary32 sqrt/div; same workload and "
                    "step count; held to a depth tolerance, not bit equality (depth error in cpu_baseline)",
            "value": cells * args.steps * world / (f["ms"] / 1e3), "unit": UNIT,
            "ms_per_step": f["ms"] / args.steps, "gpu_launches": int(f["launches"]),
            "roofline": {"bound": "hbm", "achieved": f_ach, "peak": peak, "unit": "GB/s", "frac": f_ach / peak,
                         "kernel": "gsw_fast::dense_march_kernel<float,true>", "kernel_ms": f["kern_ms"],
                         "peak_source": peak_kind},
            "issue": issue_roofline("dense_fast", cells, f["kern_ms"], f["clocks"]),
            "clocks": f["clocks"], "launch_shape": f["shape"]}
    if rank == 0 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(args)
    if world == 1 and not args.no_extras:
        out.update(extras(args))
    return out


def extras(args):
    """The rest of the metric on one GPU, each with its own workload and clock record:
    `batched` (64-member ensemble vs a loop of the plain solver, one simulated hour),
    `adjoint` (reverse step / forward step of the calibration case), `compressed` (the
    rain-on-terrain case on the compressed mesh, dense/compressed residual identity) and
    `tidal` (640 M everywhere-wet cells on the compressed mesh)."""
    import argparse as _ap
    import torch
    out = {}
    t0 = time.perf_counter()
    e = run_ensemble(args)
    out["batched"] = {
        "what": f"{e['members']} uneven members (sides log-uniform 256-4096, active 0.3-0.9, triangular "
                f"hyetographs, Manning scale 0.7-1.3), {e['t_end_s']:g} simulated s each, one persistent "
                f"launch per step in CUDA graphs vs a loop of the plain compressed solver over the same members",
        "value": e["value"], "unit": UNIT, "plain_loop_value": e["plain_loop_value"],
        "ratio": e["speedup_vs_plain_loop"], "target": ">= 3x", "target_met": e["speedup_vs_plain_loop"] >= 3.0,
        "ms_batched": e["ms_batched"], "ms_plain_loop": e["ms_plain_loop"],
        "active_cells": e["active_total"], "steps_per_member": e["steps_per_member"],
        "identical_steps_to_plain": e["identical_steps_to_plain"], "gpu_launches": e["gpu_launches"],
        "clocks_batched": e["clocks_batched"], "clocks_plain_loop": e["clocks_plain_loop"],
        "schedule": e["schedule"], "seconds": time.perf_counter() - t0}
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    a = run_adjoint(args, caps=(8,))
    out["adjoint"] = {
        "what": a["config"]["workload"], "ratio": a["value"], "unit": "reverse step / forward step",
        "target": "<= 4x", "target_met": a["value"] <= 4.0,
        "forward_ms_per_step": a["forward_ms_per_step"], "reverse_ms_per_step": a["reverse_ms_per_step"],
        "recompute_steps": a["recompute_steps"], "recompute_ms": a["recompute_ms"],
        "total_gradient_cost_in_forward_passes": a["total_gradient_cost_in_forward_passes"],
        "max_live_snapshots": a["max_live_snapshots"], "clocks_forward": a["clocks_forward"],
        "clocks_sweep": a["clocks_sweep"], "seconds": time.perf_counter() - t0}
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    c = run_compressed(_ap.Namespace(**{**vars(args), "steps": max(args.steps, 200)}))
    out["compressed"] = {k: c[k] for k in ("value", "unit", "steps", "ms_per_step", "config",
                                           "residual_bit_identical_to_dense", "residual_nonzero_fraction",
                                           "roofline", "clocks", "gpu_launches", "launch_shape")}
    out["compressed"]["seconds"] = time.perf_counter() - t0
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    t = run_tidal(_ap.Namespace(**{**vars(args), "steps": max(args.steps, 200)}))
    out["tidal"] = {k: t[k] for k in ("value", "unit", "steps", "ms_per_step", "config", "roofline", "issue",
                                      "clocks", "gpu_launches", "launch_shape", "build_s")}
    out["tidal"]["seconds"] = time.perf_counter() - t0
    torch.cuda.empty_cache()
    return out


def run_split(args, rank, world):
    """``--split``: ONE n x n rain-on-terrain domain cut into ``world`` row strips
    (``Solver2D(comm=...)``): every step each rank fills its seam ghosts from its
    neighbours and all ranks take the dt of the largest wave speed. Strong scaling:
    ``value`` is the whole domain's cell-updates/s over the slowest rank's time."""
    import torch
    import torch.distributed as dist
    from geoswe_b200.partition import block_of
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)) % torch.cuda.device_count())
    n = args.n
    z, cls = build_case(n)
    dims = [world, 1]
    block = block_of(n, n, dims, (rank, 0))
    s = make_solver(z, cls, n, block=block, comm=dist.group.WORLD if world > 1 else None, dims=dims)
    s.run(t_end=1e12, max_steps=args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = Clocks(int(os.environ.get("LOCAL_RANK", 0)) % torch.cuda.device_count())
    clk.start()
    l0 = s.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    steps = s.run(t_end=1e12, max_steps=args.steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    assert steps == args.steps, (steps, args.steps)
    backend = dist.get_backend() if world > 1 else "none"
    if world > 1:
        ms = max_over_ranks(ms, "cuda" if backend == "nccl" else "cpu")
    cfg = dense_config(n, world)
    cfg["parallelism"] = f"row strips x{world}: halo exchange + wave-speed all-reduce ({backend})"
    gpus = min(world, torch.cuda.device_count())
    return {"metric": METRIC, "value": n * n * steps / (ms / 1e3), "unit": UNIT, "n_gpus": gpus, "ranks": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg, "gpu_launches": int(s.kernel_launches - l0),
            "halo_exchanges": int(s.halo.exchanges) if s.halo is not None else 0,
            "block": list(block), "clocks": clocks, "mode": "split"}


def time_step_kernel(s, reps=20):
    """Average duration of the fused dense step kernel alone (CUDA events on its stream),
    on scratch copies of the state the timed run ended in, with the solver's launch shape."""
    from geoswe_b200.autotune import time_dense_step
    return time_dense_step(s, reps=reps, tile_rows=s._tile_rows, warps=s._warps,
                           min_blocks=s._min_blocks, dt=s.last_dt)


def run_e2e(args, z, cls, n, world=1):
    """Public API from host buffers: construct (H2D of state, bed, classes), run the
    timed steps, read the depth back (D2H), all inside the timed region; with several
    ranks, the whole job's cell-updates over the slowest rank's time. The host arrays
    sit in page-locked memory, as a pipeline feeding the solver holds them (allocated
    and filled before the timed region). One untimed call of the same path comes first,
    as the warm-up steps do for the device-resident measurement."""
    import torch
    q0 = torch.zeros((3, n, n), dtype=torch.float32).pin_memory().numpy()
    zb = torch.from_numpy(np.ascontiguousarray(z, dtype=np.float32)).pin_memory().numpy()
    clsp = torch.from_numpy(np.ascontiguousarray(np.pad(cls, 2, mode="edge"))).pin_memory().numpy()
    hout = torch.empty((n, n), dtype=torch.float32).pin_memory().numpy()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for timed in (False, True):
        torch.cuda.synchronize()
        e0.record()
        s = make_solver(zb, None, n, q0=q0, clsp=clsp)
        s.run(t_end=1e12, max_steps=args.steps if timed else max(args.warmup, 1))
        h = s.depth(out=hout)
        e1.record()
        torch.cuda.synchronize()
        del s
    ms = e0.elapsed_time(e1)
    h2d = q0.nbytes + zb.nbytes + clsp.nbytes
    d2h = h.nbytes
    if world > 1:
        ms = max_over_ranks(ms, "cuda")
    return {"value": n * n * args.steps * world / (ms / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "ms": ms, "copies_declared": True,
            "what": "Solver2D(page-locked host arrays: state, bed, padded classes) + run(steps) + "
                    "depth(out=page-locked); bytes per step = total / steps"}


def build_member(spec, brick_h=16, device="cuda", arith="exact"):
    """One member of the uneven ensemble as a CompressedSolver (inputs generated on the GPU)."""
    import torch
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import (MANNING_CLASSES, fractal_bed_device, triangular_hyetograph,
                                       voronoi_classes_device)
    nx, ny = spec["nx"], spec["ny"]
    z = fractal_bed_device(nx, ny, 3.0, seed=spec["seed"], device=device)
    thr = torch.kthvalue(z.reshape(-1).cpu(), max(1, int(spec["frac"] * nx * ny))).values.item()
    mask = (z <= thr).cpu().numpy()
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    cls = voronoi_classes_device(nx, ny, seed=spec["seed"], device=device).cpu().numpy()
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=3.0, dy=3.0, ngh=2),
                 Config(bc_x="fall", bc_y="fall", friction="manning", arith=arith),
                 np.zeros((3, nx, ny), np.float32), z.cpu().numpy(), track_max_depth=False)
    s.set_inside_mask(mask)
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES * spec["scale"])
    cs = CompressedSolver.from_dense(s, brick_h=brick_h)
    del s
    t, r = triangular_hyetograph(spec["peak"], spec["t_peak"])
    cs.set_rain(RainfallForcing(time_s=t, rate_mm_h=r))
    return cs


def run_ensemble(args):
    """Batched ensemble vs looping the plain compressed solver over the same members, for
    the same simulated window; cell-updates/s = sum over members of active cells x steps.
    The members are built once: the ensemble copies their initial states into its own
    storage, the plain loop then runs the members themselves. Both timed regions include
    their own CUDA-graph captures, each with its own tuned launch shape, and each has
    its clock record."""
    import torch
    from geoswe_b200 import autotune
    from geoswe_b200.ensemble import Ensemble
    from geoswe_b200.synthetic import ensemble_specs
    torch.cuda.set_device(0)
    specs = ensemble_specs(n_members=args.members, seed=0)
    t_end = args.ens_t_end
    # warm-up: context, library and capture paths on the smallest member
    small = min(specs, key=lambda sp: sp["nx"] * sp["ny"])
    build_member(small, arith=args.arith).run(t_end=t_end, max_steps=max(args.warmup, 3))
    Ensemble([build_member(small, arith=args.arith), build_member(small, arith=args.arith)]).run(
        t_end=t_end, max_steps=max(args.warmup, 3), window=8)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    members = [build_member(sp, arith=args.arith) for sp in specs]
    ens = Ensemble(members, warps=args.ens_warps, grid=args.ens_grid)      # copies the initial states
    ens.min_blocks, ens.segments = args.ens_min_blocks, args.ens_segments
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    loop_shape = None
    if not args.no_tune:                     # the plain solver gets its own tuned launch shape
        big = max(members, key=lambda m: m.nslots)
        best, _ = autotune.tune_flat(big, store=False)
        for m in members:       # warps per brick stay automatic: they follow each member's size
            m.warps, m.min_blocks = best["warps"], best["min_blocks"]
        loop_shape = best
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = Clocks(0)
    clk.start()
    e0.record()
    steps_loop = [m.run(t_end=t_end) for m in members]
    e1.record()
    torch.cuda.synchronize()
    clocks_loop = clk.stop()
    ms_loop = e0.elapsed_time(e1)
    loop_launches = int(sum(m.kernel_launches for m in members))
    work = sum(m.N_active * n for m, n in zip(members, steps_loop))
    for m in members:                        # the ensemble starts the members at t = 0 again
        m.t, m.nsteps = 0.0, 0
    tune = None
    if not args.no_tune and args.ens_warps == 0 and args.ens_grid == 0:
        best, table = autotune.tune_ensemble(ens, t_end)
        tune = {"best": best, "table": table}
    n0 = ens.kernel_launches
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.start()
    e0.record()
    steps_ens = ens.run(t_end=t_end, window=args.ens_window)
    e1.record()
    torch.cuda.synchronize()
    clocks_ens = clk.stop()
    ms_ens = e0.elapsed_time(e1)
    out = {"metric": METRIC + " [batched ensemble]", "value": work / (ms_ens / 1e3), "unit": UNIT,
           "n_gpus": 1, "members": len(specs), "cells_total": int(sum(sp["nx"] * sp["ny"] for sp in specs)),
           "active_total": int(sum(ens.active_cells)), "t_end_s": t_end,
           "steps_per_member": {"min": int(min(steps_ens)), "max": int(max(steps_ens)),
                                "sum": int(sum(steps_ens))},
           "ms_batched": ms_ens, "ms_plain_loop": ms_loop,
           "plain_loop_value": work / (ms_loop / 1e3), "speedup_vs_plain_loop": ms_loop / ms_ens,
           "identical_steps_to_plain": bool(steps_ens == steps_loop),
           "gpu_launches": int(ens.kernel_launches - n0), "gpu_launches_plain_loop": loop_launches,
           "clocks_batched": clocks_ens, "clocks_plain_loop": clocks_loop,
           "schedule": {"warps": ens.warps or 4, "grid": ens.grid, "min_blocks": ens.min_blocks,
                        "segments": ens.segments or 1,
                        "brick_h": ens.brick_h}, "autotune": tune, "plain_loop_shape": loop_shape,
           "build_s": build_s, "dtype": "f32", "arith": args.arith, "data": "synthetic"}
    return out


def run_adjoint(args, caps=(0, 6, 8)):
    """Calibration gradients on the compressed mesh (fp32): a 2048 x 2048 fractal terrain
    with ~70 % active cells, 4 Manning classes, rain 40 mm/h x scale, a point inlet with a
    16-knot hydrograph (20 m^3/s peak), 32 gauges, loss over the last 1000 of 3000 steps
    against a run with n x 1.2 and rain x 0.9, 55 snapshots of binomial checkpointing.
    The reported value is the cost of one reverse step over one forward step (both as
    the driver runs them, device time); recomputation is reported beside it. `caps`:
    the reverse kernels' register caps timed on the full sweep (the fastest is kept)."""
    import torch
    from geoswe_b200.adjoint import FlatAdjoint
    from geoswe_b200.synthetic import calibration_case
    from geoswe_b200.adjoint import Inlet
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    case = calibration_case(args.adj_n, seed=0, base_q=0.5, inlet_gauges=4)
    build_s = time.perf_counter() - t0
    cs = case["cs"]

    def problem(inlet):
        return FlatAdjoint(cs, gauges=case["gauges"], n_steps=args.adj_steps, window=args.adj_window,
                           snapshots=args.adj_snapshots, dtype="float32", rain_times=case["rain_times"],
                           rain_base=case["rain_base"], inlet=inlet)

    # the hydrograph's 16 knots span the simulated time of the N steps (probe run first)
    prob = problem(case["inlet"])
    prob.set_params(case["n_tab"], 1.0, case["knots"])
    prob.forward(snapshots=False)
    t_sim = prob.t_end
    inl = case["inlet"]
    kt = np.linspace(0.0, t_sim, len(inl.t_knots))
    k0 = np.maximum(0.5, 20.0 * (1.0 - np.abs(kt - t_sim / 3.0) / (t_sim / 3.0)))
    prob = problem(Inlet(ghost=inl.ghost, nbr=inl.nbr, normal=inl.normal, ds=inl.ds, t_knots=kt))
    n0 = case["n_tab"]
    prob.set_params(n0 * 1.2, 0.9, k0)
    target = prob.forward(snapshots=False).cpu().numpy()
    prob.set_params(n0, 1.0, k0)
    prob.forward(snapshots=False)                     # records the base dt schedule
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.start()
    e0.record()
    prob.forward(replay=True, snapshots=False)
    e1.record()
    torch.cuda.synchronize()
    clocks_fwd = clk.stop()
    fwd_ms = e0.elapsed_time(e1)
    e0.record()
    prob.forward()                                     # recording pass that keeps snapshots
    e1.record()
    torch.cuda.synchronize()
    rec_ms = e0.elapsed_time(e1)
    loss = prob.loss(target)
    # the reverse kernels' register cap, tried on the full sweep (the gradients must not change)
    sweeps = {}
    for i, mb in enumerate(caps):
        prob.adj_min_blocks = mb
        if i:
            prob.forward()                             # the sweep uses up the snapshots
            torch.cuda.synchronize()
        l0 = prob.kernel_launches
        clk = Clocks(0)
        clk.start()
        e0.record()
        g = prob.gradients(target, timing=True)
        e1.record()
        torch.cuda.synchronize()
        tm = dict(prob.timing)
        sweeps[mb] = dict(grad_ms=e0.elapsed_time(e1), tm=tm, g=g, launches=int(prob.kernel_launches - l0),
                          rev_step=tm["reverse_ms"] / max(tm["reverse_steps"], 1), clocks=clk.stop())
    ref_g = sweeps[caps[0]]["g"]
    for mb, sw in sweeps.items():       # equal up to the order of the per-class atomic sums
        assert torch.allclose(sw["g"][0], ref_g[0], rtol=1e-6, atol=0) and abs(sw["g"][1] - ref_g[1]) <= \
            1e-6 * abs(ref_g[1]) and torch.allclose(sw["g"][2], ref_g[2], rtol=1e-6, atol=1e-12), mb
    best_mb = min(sweeps, key=lambda k: sweeps[k]["rev_step"])
    best = sweeps[best_mb]
    gn, gs, gk = best["g"]
    grad_ms, tm = best["grad_ms"], best["tm"]
    N = prob.N
    fwd_step = fwd_ms / N
    rev_step = best["rev_step"]
    cells = int(cs.N_active)
    return {"metric": METRIC + " [adjoint/forward]", "value": rev_step / fwd_step, "unit": "x (reverse step / forward step)",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"calibration, compressed {args.adj_n}x{args.adj_n}, {cells} active cells, "
                                   f"{N} steps, loss over the last {prob.K}, {prob.G} gauges, 4 Manning classes, "
                                   f"rain scale, {len(k0)} inlet knots, {prob.S} snapshots"},
            "forward_ms_per_step": fwd_step, "reverse_ms_per_step": rev_step,
            "forward_cell_updates_per_s": cells / (fwd_step / 1e3),
            "recompute_steps": tm["recompute_steps"], "recompute_ms": tm["recompute_ms"],
            "recording_pass_ms": rec_ms, "gradient_sweep_ms": grad_ms,
            "total_gradient_cost_in_forward_passes": (rec_ms + grad_ms) / fwd_ms,
            "max_live_snapshots": prob.max_snapshots, "gpu_launches_sweep": best["launches"],
            "reverse_register_cap": {"chosen": best_mb, "reverse_ms_per_step": {str(k): v["rev_step"]
                                                                                for k, v in sweeps.items()}},
            "clocks_forward": clocks_fwd, "clocks_sweep": best["clocks"],
            "loss": loss, "grad_n": [float(x) for x in gn.cpu()], "grad_rain_scale": gs,
            "grad_knots": [float(x) for x in gk], "knot_times_s": [float(x) for x in kt],
            "knot_values": [float(x) for x in k0], "simulated_s": prob.t_end, "build_s": build_s}


def run_dambreak(args):
    """The reference's own CPU-runnable case: circular dam break on a dense 512 x 512
    grid, dx = 1 m, flat bed, h = 2 m inside r < 64 cells and 0.5 m outside, walls, no
    friction, CFL 0.5, 500 steps. GPU throughput (exact and fast arithmetic), each
    run's depth error against a binary64 run of the same scheme on the GPU (the
    binary64 kernels equal the C oracle bit for bit), and the reference's NumPy CPU
    path timed over a bounded window of the same run."""
    import torch
    from geoswe_b200 import Config, Mesh2D, Solver2D
    from geoswe_b200.synthetic import dam_break
    torch.cuda.set_device(0)
    n, steps = args.db_n, args.db_steps
    q0, bed = dam_break(n)
    res = {}
    for name, dtype, arith in (("exact", "float32", "exact"), ("fast", "float32", "fast"), ("fp64", "float64", "exact")):
        s = Solver2D(Mesh2D(nx=n, ny=n, dx=1.0, dy=1.0, ngh=2),
                     Config(bc_x="wall", bc_y="wall", cfl=0.5, h_min=1e-6, dtype=dtype, arith=arith), q0, bed)
        n_err = s.run(t_end=args.db_t_end)                       # the run compared with binary64
        h = np.asarray(s.depth(), np.float64)
        t_sim = s.t
        s2 = Solver2D(Mesh2D(nx=n, ny=n, dx=1.0, dy=1.0, ngh=2),
                      Config(bc_x="wall", bc_y="wall", cfl=0.5, h_min=1e-6, dtype=dtype, arith=arith), q0, bed)
        s2.run(t_end=1e12, max_steps=args.warmup, window=s2._window_size())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        k = s2.run(t_end=1e12, max_steps=steps)
        e1.record()
        torch.cuda.synchronize()
        res[name] = dict(h=h, t=t_sim, n_err=n_err, ms=e0.elapsed_time(e1), steps=k)
    h64 = res["fp64"]["h"]
    err = lambda h: {"max_m": float(np.abs(h - h64).max()), "rmse_m": float(np.sqrt(np.mean((h - h64) ** 2)))}
    from oracle import numpy_ref
    cpu_steps = min(steps, args.cpu_steps * 5)
    ref = numpy_ref.NumpySolver2D(np.pad(q0.astype(np.float32), ((0, 0), (2, 2), (2, 2))),
                                  np.zeros((n + 4, n + 4), np.float32), 2, 1.0, 1.0, kinds=("wall",) * 4)
    ref.run(t_end=1e12, max_steps=2)
    t0 = time.perf_counter()
    ref.run(t_end=1e12, max_steps=cpu_steps)
    cpu_s = time.perf_counter() - t0
    cells = n * n
    ex, fa = res["exact"], res["fast"]
    return {"metric": METRIC + " [dam break]", "value": cells * steps / (ex["ms"] / 1e3), "unit": UNIT,
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ex["ms"] / steps,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"circular dam break {n}x{n}, dx=1 m, flat bed, h=2 m in r<64 cells, 0.5 m "
                                   f"outside, walls, no friction, CFL 0.5, {steps} steps, fp32"},
            "fast_arith": {"value": cells * steps / (fa["ms"] / 1e3), "ms_per_step": fa["ms"] / steps},
            "depth_error_vs_fp64": {"exact": err(ex["h"]), "fast": err(fa["h"]), "t_s": ex["t"],
                                    "steps": {k: int(v["n_err"]) for k, v in res.items()}},
            "cpu_baseline": {"value": cells * cpu_steps / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"reference NumPy path (oracle/numpy_ref.py), the same {n}x{n} run, "
                                       f"{cpu_steps} steps after 2, fp32, 1 core"}}


def run_compressed(args):
    """The rain-on-terrain case on the compressed mesh: active set z < 60th percentile of
    the bed dilated by 8 cells (cross), packed from the dense solver; the dense and
    compressed residuals compared bit for bit at a wet state (after the warm-up), then
    the compressed run timed."""
    import torch
    from geoswe_b200 import autotune
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import dilate_cross
    torch.cuda.set_device(0)
    n = args.n
    z, cls = build_case(n)
    inside = dilate_cross(z < np.percentile(z, 60.0), 8)
    inside[:3, :] = inside[-3:, :] = False
    inside[:, :3] = inside[:, -3:] = False
    s = make_solver(z, cls, n, arith=args.arith)
    s.set_inside_mask(inside)
    s.run(t_end=1e12, max_steps=max(args.warmup, 3))       # a wet state (rain on the dry start)
    s.apply_bc()
    r_dense = s.residual()
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        cs = CompressedSolver.from_dense(s, brick_h=args.brick_h)
    del s
    torch.cuda.empty_cache()
    from geoswe_b200 import RainfallForcing
    cs.set_rain(RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0]))
    r_flat = cs.residual()
    act = torch.from_numpy(cs.is_active != 0).to(r_flat.device)
    ij = torch.from_numpy(cs.ij_active).to(r_flat.device)
    identical = all(bool(torch.equal(r_flat[c][act], r_dense[c][ij[act, 0], ij[act, 1]])) for c in range(3))
    wet = float((r_dense[0] != 0).float().mean())
    del r_dense, r_flat
    tune = None
    if args.flat_shape:
        cs.warps, cs.min_blocks, cs.segments = (int(v) for v in args.flat_shape.split(","))
    elif not args.no_tune:
        best, table = autotune.tune_flat(cs, reps=4)
        tune = {"best": best}
    cs.run(t_end=1e12, max_steps=args.warmup, window=cs._window_size())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = cs.kernel_launches
    clk = Clocks(0)
    clk.start()
    e0.record()
    steps = cs.run(t_end=1e12, max_steps=args.steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    torch.cuda.nvtx.range_push("kernel_timing")        # the launches an ncu capture targets
    kern_ms = autotune.time_flat_step(cs, reps=args.kernel_reps)
    torch.cuda.nvtx.range_pop()
    cells = int(cs.N_active)
    peak, peak_kind = _peaks()
    achieved = 38.0 * cells / (kern_ms / 1e3) / 1e9
    return {"metric": METRIC + " [compressed rain-on-terrain]", "clocks": clocks, "value": cells * steps / (ms / 1e3), "unit": UNIT,
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "dtype": "f32", "arith": args.arith, "data": "synthetic",
            "config": {"workload": f"rain-on-terrain {n}x{n} on the compressed mesh, active z < p60 dilated 8 "
                                   f"cells, 50 mm/h, CFL 0.5, fp32",
                       "active_cells": cells, "stored_slots": int(cs.nslots), "bricks": int(cs.n_bricks),
                       "brick_h": cs.brick_h},
            "residual_bit_identical_to_dense": identical, "residual_nonzero_fraction": wet,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "kernel_ms": kern_ms, "bytes_per_cell": 38,
                         "traffic": _traffic("flat_compressed", cells)[0],
                         "traffic_from": _traffic("flat_compressed", cells)[1],
                         "peak_source": peak_kind},
            "issue": issue_roofline("flat_compressed", cells, kern_ms, None),
            "gpu_launches": int(cs.kernel_launches - l0),
            "launch_shape": {"warps": cs.warps or 4, "min_blocks": cs.min_blocks, "segments": cs.segments or "auto"},
            "autotune": tune}


def run_tidal(args):
    """Everywhere-wet throughput on the compressed mesh: 32000 x 20000 = 640 M cells, all
    active, dx = 1 m, bed 0.5 sin(2 pi x / 2000) cos(2 pi y / 1500) m, free surface 1.5 m
    plus 1 cm seeded noise, zero velocity, n = 0.03, tidal stage 1.5 + 0.3 sin(2 pi t /
    44712 s) on the x- ghost ring (one gauge, weight 1), CFL 0.5, fp32, `steps` timed
    steps. The roofline basis is 38 B per active cell (the reference's table format:
    state, bed, class, int16 neighbours, flag); the brick layout's own DRAM traffic is
    measured with ncu on a smaller all-wet case."""
    import torch
    import warnings
    from geoswe_b200 import Config, Mesh2D, Solver2D, autotune
    from geoswe_b200.compressed import CompressedSolver
    torch.cuda.set_device(0)
    nx, ny, dx = args.tidal_nx, args.tidal_ny, 1.0
    t0 = time.perf_counter()
    dev = torch.device("cuda")
    x = (torch.arange(nx, device=dev, dtype=torch.float64) + 0.5) * dx
    y = (torch.arange(ny, device=dev, dtype=torch.float64) + 0.5) * dx
    z = (0.5 * torch.sin(2 * np.pi * x / 2000.0)[:, None] * torch.cos(2 * np.pi * y / 1500.0)[None, :]).float()
    gen = torch.Generator(device=dev).manual_seed(0)
    eta = 1.5 + 0.01 * torch.randn((nx, ny), generator=gen, device=dev, dtype=torch.float32)
    h = torch.clamp(eta - z, min=0.0)
    del eta
    q0 = np.zeros((3, nx, ny), np.float32)
    q0[0] = h.cpu().numpy()
    zh = z.cpu().numpy()
    del h, z, x, y
    torch.cuda.empty_cache()
    cfg = Config(bc_x="wall", bc_y="wall", friction="manning", manning_n=0.03, cfl=0.5, arith=args.arith)
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=2), cfg, q0, zh, track_max_depth=False)
    del q0, zh
    s.apply_bc()
    ngh = s.mesh.ngh
    ri = np.repeat(np.arange(ngh), s.nyp)
    rj = np.tile(np.arange(s.nyp), ngh)
    rbed = s._b[:ngh, : s.nyp].reshape(-1).cpu().numpy().astype(np.float32)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        cs = CompressedSolver.from_dense(s, track_max_depth=False, brick_h=args.brick_h)
    del s
    torch.cuda.empty_cache()
    t_c = np.arange(0.0, 3600.0 + 60.0, 60.0)
    stage = (1.5 + 0.3 * np.sin(2 * np.pi * t_c / 44712.0)).astype(np.float32)[None, :]
    cs.set_ring(dict(i=ri, j=rj, bed=rbed, wg=np.ones((ri.size, 1), np.float32), NG=1, n=int(ri.size),
                     t_common=t_c, stage_all=stage))
    build_s = time.perf_counter() - t0
    if args.flat_shape:
        cs.warps, cs.min_blocks, cs.segments = (int(v) for v in args.flat_shape.split(","))
    cs.run(t_end=1e12, max_steps=args.warmup)
    tune = None
    if not args.no_tune and not args.flat_shape:
        best, table = autotune.tune_flat(cs, reps=4)
        tune = {"best": best, "table": table}
    cs.run(t_end=1e12, max_steps=args.warmup, window=cs._window_size())   # captures the timed window's graph
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = cs.kernel_launches
    e0.record()
    steps = cs.run(t_end=1e12, max_steps=args.steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    launches = cs.kernel_launches - l0
    torch.cuda.nvtx.range_push("kernel_timing")        # the launches an ncu capture targets
    kern_ms = autotune.time_flat_step(cs, reps=args.kernel_reps)
    torch.cuda.nvtx.range_pop()
    cells = int(cs.N_active)
    peak, peak_kind = _peaks()
    achieved = 38.0 * cells / (kern_ms / 1e3) / 1e9
    stored_bytes = 29.0 * cs.nslots                      # q in + bed + flag + q out per slot
    return {"metric": METRIC + " [compressed, everywhere wet]", "value": cells * steps / (ms / 1e3), "unit": UNIT,
            "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps,
            "higher_is_better": True, "dtype": "f32", "arith": args.arith, "data": "synthetic",
            "config": {"workload": f"tidal everywhere-wet compressed {nx}x{ny}, dx=1 m, sinusoidal bed, "
                                   f"n=0.03, tidal stage on the x- ring, CFL 0.5, fp32",
                       "active_cells": cells, "stored_slots": int(cs.nslots), "bricks": int(cs.n_bricks),
                       "brick_h": cs.brick_h, "l2": "inputs larger than L2 (no flush)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": _traffic("flat_tidal", cells)[0],
                         "traffic_from": _traffic("flat_tidal", cells)[1],
                         "kernel": "flat_march_kernel<float,1>",
                         "kernel_ms": kern_ms, "bytes_per_cell": 38, "peak_source": peak_kind,
                         "brick_bytes_GBs": stored_bytes / (kern_ms / 1e3) / 1e9},
            "issue": issue_roofline("flat_tidal", cells, kern_ms, clocks) if args.arith == "exact" else None,
            "gpu_launches": int(launches), "clocks": clocks, "build_s": build_s, "simulated_s": cs.t,
            "launch_shape": {"warps": cs.warps or 4, "min_blocks": cs.min_blocks, "segments": cs.segments or 1},
            "autotune": tune}


def cpu_baseline(args):
    """The reference's CPU path (its NumPy solver, restated in oracle/numpy_ref.py) on a
    bounded sample of the same workload, on this host's cores."""
    try:
        from oracle import numpy_ref
    except Exception as e:                      # pragma: no cover
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "port", "sample": f"unavailable: {e}"}
    out = numpy_ref.time_rain_on_terrain(n=args.cpu_n, steps=args.cpu_steps)
    if args.err_n > 0:
        out["depth_error_vs_fp64"] = fp64_depth_error(args.err_n, args.err_t_end)
    return out


def fp64_depth_error(n, t_end):
    """Depth error of the product (fp32, GPU) against an fp64 run of the same scheme on
    the CPU (the reference's NumPy path, restated in the oracle), on an n x n sample of
    the rain-on-terrain case run to the same simulated time."""
    import torch
    from oracle import numpy_ref
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.synthetic import MANNING_CLASSES, fractal_bed, voronoi_classes
    t0 = time.perf_counter()
    ref = numpy_ref._rain_on_terrain_solver(n, dtype=np.float64)
    steps64 = ref.run(t_end=t_end)
    z = fractal_bed(n, n, 3.0, seed=0).astype(np.float32)
    cls = voronoi_classes(n, n, seed=0)
    cfg = Config(bc_x="wall", bc_y="wall", bc={"x+": "fall"}, friction="manning",
                 rainfall_forcing=RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0]))
    s = Solver2D(Mesh2D(nx=n, ny=n, dx=3.0, dy=3.0, ngh=2), cfg, np.zeros((3, n, n), np.float32), z)
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES)
    steps32 = s.run(t_end=t_end)
    torch.cuda.synchronize()
    h32 = s.depth().astype(np.float64)
    h64 = ref.q[0][2:-2, 2:-2]
    cfg_f = Config(bc_x="wall", bc_y="wall", bc={"x+": "fall"}, friction="manning", arith="fast",
                   rainfall_forcing=RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0]))
    sf = Solver2D(Mesh2D(nx=n, ny=n, dx=3.0, dy=3.0, ngh=2), cfg_f, np.zeros((3, n, n), np.float32), z)
    sf.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES)
    steps_f = sf.run(t_end=t_end)
    df = sf.depth().astype(np.float64) - h64
    # the reference's NumPy fp32 path (it accumulates the bed source in float64)
    ref32 = numpy_ref._rain_on_terrain_solver(n, dtype=np.float32)
    steps_r32 = ref32.run(t_end=t_end)
    hr32 = ref32.q[0][2:-2, 2:-2].astype(np.float64)
    d, dr = h32 - h64, hr32 - h64
    return {"case": f"rain-on-terrain {n}x{n}, t = {t_end:g} s", "max_m": float(np.abs(d).max()),
            "rmse_m": float(np.sqrt(np.mean(d * d))), "mean_depth_m": float(h64.mean()),
            "steps_fp32_gpu": int(steps32), "steps_fp64_cpu": int(steps64),
            "reference_numpy_fp32_vs_fp64": {"max_m": float(np.abs(dr).max()),
                                           "rmse_m": float(np.sqrt(np.mean(dr * dr))), "steps": int(steps_r32)},
            "fast_arith_vs_fp64": {"max_m": float(np.abs(df).max()), "rmse_m": float(np.sqrt(np.mean(df * df))),
                                   "steps": int(steps_f)},
            "seconds": time.perf_counter() - t0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gsw", choices=["gsw", "reference"])
    ap.add_argument("--n", "--grid", dest="n", type=int, default=8192,
                    help="grid side (--grid under torchrun, whose own options --n would abbreviate)")
    ap.add_argument("--kernel-reps", type=int, default=20)
    ap.add_argument("--cpu-n", type=int, default=512)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fast", action="store_true", help="skip the fast-arithmetic measurement")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched / adjoint / compressed / tidal objects of the default line")
    ap.add_argument("--dense-arith", default="exact", choices=["exact", "portable"],
                    help="arithmetic of the headline dense measurement (portable: Manning power by the "
                         "Newton iteration instead of powf)")
    ap.add_argument("--arith", default="exact", choices=["exact", "fast", "portable"],
                    help="step arithmetic of the tidal and ensemble cases")
    ap.add_argument("--exact-shape", default="", help="dense launch shape 'tile_rows,warps,min_blocks' (no tuning)")
    ap.add_argument("--fast-shape", default="", help="the same for the fast arithmetic")
    ap.add_argument("--flat-shape", default="", help="compressed-mesh launch shape 'warps,min_blocks,segments' "
                                                     "(no tuning)")
    ap.add_argument("--err-n", type=int, default=96, help="fp64 depth-error sample size (0: skip)")
    ap.add_argument("--err-t-end", type=float, default=600.0)
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--case", default="dense", choices=["dense", "ensemble", "adjoint", "tidal", "dambreak",
                                                        "compressed"])
    ap.add_argument("--db-n", type=int, default=512)
    ap.add_argument("--db-steps", type=int, default=500)
    ap.add_argument("--db-t-end", type=float, default=50.0, help="simulated time of the fp64 comparison")
    ap.add_argument("--brick-h", type=int, default=16, help="rows per brick of the compressed and tidal cases")
    ap.add_argument("--tidal-nx", type=int, default=32000)
    ap.add_argument("--tidal-ny", type=int, default=20000)
    ap.add_argument("--adj-n", type=int, default=2048)
    ap.add_argument("--adj-steps", type=int, default=3000)
    ap.add_argument("--adj-window", type=int, default=1000)
    ap.add_argument("--adj-snapshots", type=int, default=55)
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--ens-t-end", type=float, default=3600.0)
    ap.add_argument("--ens-window", type=int, default=32)
    ap.add_argument("--ens-warps", type=int, default=0)
    ap.add_argument("--ens-grid", type=int, default=0)
    ap.add_argument("--ens-min-blocks", type=int, default=0, help="ensemble register cap (with --ens-warps/--ens-grid)")
    ap.add_argument("--ens-segments", type=int, default=0, help="ensemble warps per brick (0: automatic)")
    ap.add_argument("--split", action="store_true",
                    help="one domain cut into row strips over the ranks (strong scaling) instead of replicas")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process group of --split (gloo: host-staged, for several ranks on one GPU)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        from oracle import numpy_ref
        out = numpy_ref.reference_arm(args, METRIC, UNIT, config=dense_config(args.n, world))
        print(json.dumps(out), flush=True)
        return 0
    if args.case in ("ensemble", "adjoint", "tidal", "dambreak", "compressed"):
        if rank == 0:
            out = {"ensemble": run_ensemble, "adjoint": run_adjoint, "tidal": run_tidal, "dambreak": run_dambreak,
                   "compressed": run_compressed}[args.case](args)
            print(json.dumps(out), flush=True)
        return 0
    if args.split:
        import datetime
        import torch
        if world > 1:
            torch.distributed.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=300))
        out = run_split(args, rank, world)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    if world > 1:
        import torch
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_gsw(args, rank, world)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
