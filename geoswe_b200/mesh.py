"""Structured mesh (the reference's Mesh2D, geoswe/mesh.py:46-87)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Mesh2D:
    """Uniform 2D cell-centred Cartesian mesh: ``nx x ny`` cells of ``dx x dy`` with
    ``ngh`` ghost layers on every side. The fused step needs ``ngh >= 2``."""
    nx: int
    ny: int
    dx: float
    dy: float
    x0: float = 0.0
    y0: float = 0.0
    ngh: int = 4

    def __post_init__(self):
        if int(self.nx) < 1 or int(self.ny) < 1:
            raise ValueError(f"Mesh2D: nx, ny must be >= 1 (got {self.nx}, {self.ny})")
        if not (float(self.dx) > 0.0 and float(self.dy) > 0.0):
            raise ValueError(f"Mesh2D: dx, dy must be positive (got {self.dx}, {self.dy})")
        self.nx, self.ny, self.ngh = int(self.nx), int(self.ny), int(self.ngh)
        self.x = self.x0 + (np.arange(self.nx) + 0.5) * self.dx
        self.y = self.y0 + (np.arange(self.ny) + 0.5) * self.dy
        self.shape = (self.nx, self.ny)

    @property
    def padded_shape(self):
        return (self.nx + 2 * self.ngh, self.ny + 2 * self.ngh)

    def interior(self, arr):
        """Strip the ghost layers of one padded 2-D field."""
        if arr.ndim != 2:
            raise ValueError(f"Mesh2D.interior expects a 2-D scalar field, got ndim={arr.ndim}")
        g = self.ngh
        return arr[g:-g, g:-g] if g > 0 else arr

    def pad(self, arr):
        """Zero-pad one (nx, ny) field with ngh ghost layers."""
        arr = np.asarray(arr)
        if arr.ndim != 2:
            raise ValueError(f"Mesh2D.pad expects a 2-D scalar field, got ndim={arr.ndim}")
        out = np.zeros(self.padded_shape, dtype=arr.dtype)
        out[self.ngh:self.ngh + self.nx, self.ngh:self.ngh + self.ny] = arr
        return out
