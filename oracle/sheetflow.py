"""Exact steady sheet flow on a rained plane (test infrastructure).

A restatement of the reference's known-answer case (benchmark/sheetflow_plane/
exact_profile.py:37-51, the paper's Sect. 5.5, Eq. 16): uniform rain r on a plane of
slope S fixes q(x) = r x by mass balance from the divide; the steady momentum balance
d/dx(q^2/h + g h^2/2) = g h (S - n^2 q^2 / h^(10/3)) has no closed form and is solved
by relaxing the fixed point h = (n^2 q^2 / (S - dh/dx - d(q^2/h)/dx / (g h)))^(3/10)
from the kinematic profile (n r x / sqrt(S))^(3/5). The reference's published mean
errors of its own solver against this profile over x = 30..294 m
(benchmark/sheetflow_plane/README.md) are +0.75 % (22.04 mm/h, dx 3 m), +0.80 %
(348 mm/h, dx 3 m) and +0.25 % (22.04 mm/h, dx 1 m).
"""
from __future__ import annotations

import numpy as np

PUBLISHED_MEAN_ERROR = {(22.04, 3.0): 0.0075, (348.0, 3.0): 0.0080, (22.04, 1.0): 0.0025}


def plane_x(dx, n_plane=None):
    """Cell centres of the 300 m plane."""
    n_plane = n_plane if n_plane is not None else int(round(300.0 / dx))
    return (np.arange(n_plane) + 0.5) * dx


def band(dx):
    """The scored interior band, x = 30..294 m, as a slice of plane_x(dx)."""
    return slice(int(round(30.0 / dx)), int(round(294.0 / dx)))


def kinematic_profile(x, r, S=0.015, n=0.12):
    return (n * r * np.asarray(x, np.float64) / np.sqrt(S)) ** 0.6


def exact_profile(x, r, S=0.015, n=0.12, g=9.81, iters=300, relax=0.3):
    """Depth (m) of the steady gradually varied profile at the cell centres x."""
    x = np.asarray(x, np.float64)
    q = r * x
    h = kinematic_profile(x, r, S, n)
    for _ in range(iters):
        slope = S - np.gradient(h, x) - np.gradient(q * q / h, x) / (g * h)
        slope = np.maximum(slope, 1e-4)
        h = (1.0 - relax) * h + relax * (n * n * q * q / slope) ** 0.3
    return h
