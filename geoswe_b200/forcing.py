"""Rainfall and stage forcings (the reference's geoswe/forcing.py:94-377).

Both keep the reference's host-side semantics -- piecewise-constant rain selected by
``bisect_right(time_s, t) - 1`` and clamped, stage by linear interpolation clamped at
the ends -- and additionally hand their tables to the device, where the solvers
evaluate them inside the captured time loop.
"""
from __future__ import annotations

import bisect
import warnings
from dataclasses import dataclass

import numpy as np


def _require_time_order(who, time_s):
    t = np.asarray(time_s, dtype=np.float64)
    back = np.nonzero(np.diff(t) < 0.0)[0]
    if back.size:
        k = int(back[0])
        raise ValueError(f"{who}: time_s must be non-decreasing, but time_s[{k + 1}]={t[k + 1]:.6g} "
                         f"< time_s[{k}]={t[k]:.6g}")


@dataclass
class RainfallForcing:
    """Time-varying rainfall. ``rate_mm_h`` is ``(nt,)`` (uniform) or ``(nt, nx, ny)``
    (gridded); the k-th rate holds from ``time_s[k]`` to ``time_s[k+1]``."""
    time_s: np.ndarray
    rate_mm_h: np.ndarray

    def __post_init__(self):
        if isinstance(self.time_s, (list, tuple)):
            self.time_s = np.asarray(self.time_s, dtype=np.float64)
        if isinstance(self.rate_mm_h, (list, tuple)):
            self.rate_mm_h = np.asarray(self.rate_mm_h, dtype=np.float64)
        self.time_s = np.asarray(self.time_s)
        self.rate_mm_h = np.asarray(self.rate_mm_h)
        nd = int(getattr(self.rate_mm_h, "ndim", 1))
        if nd not in (1, 3):
            raise ValueError(f"RainfallForcing: rate_mm_h has shape {tuple(self.rate_mm_h.shape)}; "
                             f"it must be (nt,) or (nt, nx, ny)")
        if int(self.rate_mm_h.shape[0]) != len(self.time_s):
            raise ValueError(f"RainfallForcing: {len(self.time_s)} times but "
                             f"{int(self.rate_mm_h.shape[0])} rates; give one rate per time")
        _require_time_order("RainfallForcing", self.time_s)

    @classmethod
    def from_uniform_constant(cls, rate_mm_h: float, t_end: float = 1e9):
        return cls(time_s=np.array([0.0, t_end], dtype=np.float64),
                   rate_mm_h=np.array([rate_mm_h, rate_mm_h], dtype=np.float64))

    @property
    def gridded(self) -> bool:
        return self.rate_mm_h.ndim == 3

    def index_at(self, t: float) -> int:
        tl = self.time_s.tolist()
        idx = max(0, bisect.bisect_right(tl, float(t)) - 1)
        return min(idx, len(tl) - 1)

    def rate_at_time(self, t: float, frame_dtype=None):
        """Rate in m/s at ``t``: a float (uniform) or an (nx, ny) NumPy frame."""
        idx = self.index_at(t)
        if self.rate_mm_h.ndim == 1:
            return float(self.rate_mm_h[idx]) / 3.6e6
        frame = np.asarray(self.rate_mm_h[idx]) / 3.6e6
        if frame_dtype is not None and frame.dtype != frame_dtype:
            frame = frame.astype(frame_dtype)
        return frame

    def frames(self, frame_dtype):
        """Every rate in m/s as the solver reads it: a (nt,) table or (nt, nx, ny) frames
        (the reference's rate_at_time conversion, one frame per time)."""
        if self.rate_mm_h.ndim == 1:
            return np.array([float(r) / 3.6e6 for r in self.rate_mm_h], dtype=frame_dtype)
        out = np.empty(self.rate_mm_h.shape, dtype=frame_dtype)
        for k in range(self.rate_mm_h.shape[0]):
            out[k] = (np.asarray(self.rate_mm_h[k]) / 3.6e6).astype(frame_dtype, copy=False)
        return out


@dataclass
class StageBoundary:
    """Water-surface elevation eta(t) imposed on padded cells ``cells`` (M, 2):
    h = max(eta - bed_b, 0), hu = hv = 0, after each step."""
    cells: np.ndarray
    time_s: np.ndarray
    stage_m: np.ndarray
    bed_b: np.ndarray

    def __post_init__(self):
        if isinstance(self.time_s, (list, tuple)):
            self.time_s = np.asarray(self.time_s, dtype=np.float64)
        if isinstance(self.stage_m, (list, tuple)):
            self.stage_m = np.asarray(self.stage_m, dtype=np.float64)
        self.cells = np.asarray(self.cells)
        self.bed_b = np.asarray(self.bed_b)
        if len(self.time_s) != len(self.stage_m):
            raise ValueError(f"StageBoundary: {len(self.time_s)} times but "
                             f"{len(self.stage_m)} stage values")
        _require_time_order("StageBoundary", self.time_s)
        if self.cells.ndim != 2 or self.cells.shape[1] != 2:
            raise ValueError("StageBoundary.cells must have shape (M, 2)")
        if len(self.bed_b) != len(self.cells):
            raise ValueError("StageBoundary.bed_b must have one value per cell")

    @classmethod
    def from_mask(cls, mask, mesh, bed, time_s, stage_m):
        mask = np.asarray(mask, dtype=bool)
        bed = np.asarray(bed)
        if mask.shape != (mesh.nx, mesh.ny) or bed.shape != mask.shape:
            raise ValueError(f"StageBoundary.from_mask: mask and bed must have shape "
                             f"({mesh.nx}, {mesh.ny}); got {mask.shape} and {bed.shape}")
        return cls(cells=np.argwhere(mask) + mesh.ngh, time_s=time_s, stage_m=stage_m,
                   bed_b=bed[mask])

    def stage_at_time(self, t: float) -> float:
        tl = list(np.asarray(self.time_s, dtype=np.float64).tolist())
        sl = list(np.asarray(self.stage_m, dtype=np.float64).tolist())
        t_f = float(t)
        if t_f <= tl[0]:
            return sl[0]
        if t_f >= tl[-1]:
            return sl[-1]
        i = bisect.bisect_left(tl, t_f)
        t0, t1, s0, s1 = tl[i - 1], tl[i], sl[i - 1], sl[i]
        w = (t_f - t0) / (t1 - t0)
        return s0 + w * (s1 - s0)

    def warn_if_uncovered(self, t_end):
        tl = np.asarray(self.time_s, dtype=np.float64)
        if float(t_end) > float(tl[-1]) or 0.0 < float(tl[0]):
            warnings.warn(f"StageBoundary: the run window [0, {float(t_end):.0f}] s leaves the stage "
                          f"coverage [{tl[0]:.0f}, {tl[-1]:.0f}]; clamping to the endpoint value.",
                          RuntimeWarning, stacklevel=3)
