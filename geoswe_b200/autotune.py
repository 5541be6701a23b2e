"""Launch-shape autotuner for the fused step kernels.

The dense step's speed depends on the rows a warp walks (tile_rows), the warps per
block and the register cap (occupancy against spills); the best point depends on the
device and on how wet the grid is. `tune_dense` times each candidate with CUDA events
on scratch copies of a solver's current state (the solver itself is not advanced) and
caches the winner as JSON keyed by device name, driver version and grid size class.

Cache: $GSW_TUNE_CACHE, else ~/.cache/geoswe_b200/autotune.json.
"""
from __future__ import annotations

import ctypes as C
import itertools
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _lib as L

DENSE_SPACE = dict(tile_rows=(0, 4, 8, 16, 32, 64), warps=(2, 4, 8), min_blocks=(0, 3, 4, 5))


def _cache_path() -> Path:
    p = os.environ.get("GSW_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "geoswe_b200" / "autotune.json"


def kind(base, arith=0):
    """Cache kind of a kernel family: the fast-arithmetic kernels tune separately."""
    return base + "-fast" if int(arith) == L.ARITH_FAST else base


def _key(kind, cells):
    dev = torch.cuda.get_device_name()
    drv = torch.version.cuda or ""
    try:
        import ctypes
        v = ctypes.c_int()
        ctypes.CDLL("libcuda.so.1").cuDriverGetVersion(ctypes.byref(v))
        drv = str(v.value)
    except Exception:
        pass
    size = "small" if cells < 1 << 20 else ("medium" if cells < 1 << 24 else "large")
    return f"{kind}|{dev}|{drv}|{size}"


def load(kind, cells):
    p = _cache_path()
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(_key(kind, cells))
    except Exception:
        return None


def _store(kind, cells, entry):
    """Add an entry to the JSON cache. Best effort: processes tuning at the same time
    (one per GPU) each write their own temporary file and rename it into place; a
    process whose write fails keeps its result in memory only."""
    p = _cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        data = {}
        if p.exists():
            try:
                data = json.loads(p.read_text())
            except Exception:
                data = {}
        data[_key(kind, cells)] = entry
        tmp = p.with_name(f"{p.name}.{os.getpid()}.tmp")
        tmp.write_text(json.dumps(data, indent=1))
        os.replace(tmp, p)
    except OSError:
        pass


def time_dense_step(s, reps=10, tile_rows=0, warps=0, min_blocks=0, dt=None):
    """Mean duration (ms) of one fused dense step launch of solver `s` on scratch copies
    of its current state."""
    from .solver import _ptr, _stream
    T = s._tables()
    if dt is None:
        dt = s.cfl_dt()
    st = L.GswLoopState()
    st.t = s.t
    st.dt = float(dt)
    st.dt_f32 = float(np.float32(dt))
    state = torch.zeros(128, dtype=torch.uint8, device=s.device)
    state.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))), dtype=torch.uint8))
    bufs = [s._buf[s._cur].clone(), torch.empty_like(s._buf[s._cur])]
    maxh = None if s._max_h is None else s._max_h.clone()
    args = []
    for k in (0, 1):
        a = s._dense_args(bufs[k], bufs[1 - k], T)
        a.state = _ptr(state)
        a.lam_target = C.c_void_p(state.data_ptr() + L.GswLoopState.lam_bits.offset)
        a.max_h = _ptr(maxh)
        a.tile_rows, a.warps, a.min_blocks = int(tile_rows), int(warps), int(min_blocks)
        args.append(a)
    for k in range(2):
        L.call("gsw_dense_step", C.byref(args[k % 2]), _stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(reps):
        L.call("gsw_dense_step", C.byref(args[k % 2]), _stream())
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_dense(s, reps=8, space=None, store=True, verbose=False):
    """Time every launch shape of `space` on solver `s`; return (best, table) and cache
    the best for this device and size class."""
    space = space or DENSE_SPACE
    dt = s.cfl_dt()
    table = []
    for tr, w, mb in itertools.product(space["tile_rows"], space["warps"], space["min_blocks"]):
        ms = time_dense_step(s, reps=reps, tile_rows=tr, warps=w, min_blocks=mb, dt=dt)
        table.append(dict(tile_rows=tr, warps=w, min_blocks=mb, ms=ms))
        if verbose:
            print(f"  tile_rows={tr:3d} warps={w} min_blocks={mb}: {ms:.4f} ms", flush=True)
    best = min(table, key=lambda e: e["ms"])
    cells = s.mesh.nx * s.mesh.ny
    if store:
        _store(kind("dense", s.arith), cells, best)
    return best, table


ENSEMBLE_SPACE = dict(warps=(4, 8), blocks_per_sm=(2, 4, 8), min_blocks=(0, 3, 4), segments=(0, 1))
FLAT_SPACE = dict(warps=(2, 4, 8), min_blocks=(0, 3, 4, 5), segments=(0, 1, 2, 4))


def tune_ensemble(ens, t_end, reps=6, space=None, store=True, verbose=False):
    """Time the ensemble step for every (warps, blocks per SM, register cap) of `space` from the
    ensemble's current state (restored before every launch, so nothing advances); set
    the winner on `ens` and cache it. Returns (best, table)."""
    space = space or ENSEMBLE_SPACE
    sms = torch.cuda.get_device_properties(ens.device).multi_processor_count
    table = []
    segs = [g for g in space.get("segments", (1,)) if g == 0 or ens.brick_h % g == 0]
    for w, bps, mb, g in itertools.product(space["warps"], space["blocks_per_sm"], space.get("min_blocks", (0,)),
                                           segs):
        ms = ens.time_step(t_end, warps=w, grid=bps * sms, min_blocks=mb, segments=g, reps=reps)
        table.append(dict(warps=w, blocks_per_sm=bps, grid=bps * sms, min_blocks=mb, segments=g, ms=ms))
        if verbose:
            print(f"  warps={w} blocks/SM={bps} min_blocks={mb} segments={g}: {ms:.4f} ms", flush=True)
    best = min(table, key=lambda e: e["ms"])
    ens.warps, ens.grid, ens.min_blocks = best["warps"], best["grid"], best["min_blocks"]
    ens.segments = best["segments"]
    if store:
        _store(kind("ensemble", ens.arith), ens.nslots, best)
    return best, table


def time_flat_step(cs, reps=10, dt=None, warps=None, min_blocks=None, segments=None):
    """Mean duration (ms) of one fused flat-step launch of compressed solver `cs` on
    scratch copies of its state (the solver is not advanced), with the solver's own
    launch shape unless `warps` / `min_blocks` / `segments` are given."""
    from .solver import _ptr, _stream
    if dt is None:
        dt = getattr(cs, "last_dt", None) or 0.01
    st = L.GswLoopState()
    st.t = cs.t
    st.dt = float(dt)
    st.dt_f32 = float(np.float32(dt))
    state = torch.zeros(128, dtype=torch.uint8, device=cs.device)
    state.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))), dtype=torch.uint8))
    src = [x.clone() for x in cs._q[cs._cur]]
    dst = [torch.empty_like(x) for x in src]
    args = []
    for k in (0, 1):
        a = cs._args(src if k == 0 else dst, dst if k == 0 else src)
        a.state = _ptr(state)
        a.lam_target = C.c_void_p(state.data_ptr() + L.GswLoopState.lam_bits.offset)
        if warps is not None:
            a.warps = int(warps)
        if min_blocks is not None:
            a.min_blocks = int(min_blocks)
        if segments is not None:
            a.segments = int(segments)
        args.append(a)
    for k in range(2):
        L.call("gsw_flat_step", C.byref(args[k % 2]), _stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(reps):
        L.call("gsw_flat_step", C.byref(args[k % 2]), _stream())
    e1.record()
    torch.cuda.synchronize()
    del src, dst
    return e0.elapsed_time(e1) / reps


def tune_flat(cs, reps=6, space=None, store=True, verbose=False):
    """Time the fused flat step for every (warps, register cap, row segments per brick)
    of `space` on scratch copies of `cs`'s state; set the winner on `cs` and cache it.
    Returns (best, table)."""
    space = space or FLAT_SPACE
    table = []
    segs = [g for g in space.get("segments", (1,)) if g == 0 or cs.brick_h % g == 0]
    for w, mb, g in itertools.product(space["warps"], space["min_blocks"], segs):
        ms = time_flat_step(cs, reps=reps, warps=w, min_blocks=mb, segments=g)
        table.append(dict(warps=w, min_blocks=mb, segments=g, ms=ms))
        if verbose:
            print(f"  warps={w} min_blocks={mb} segments={g}: {ms:.4f} ms", flush=True)
    best = min(table, key=lambda e: e["ms"])
    cs.warps, cs.min_blocks, cs.segments = best["warps"], best["min_blocks"], best["segments"]
    cs._graph_cache.clear()
    if store:
        _store(kind("flat", cs.arith), cs.nslots, best)
    return best, table
