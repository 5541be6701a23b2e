"""Solver configuration (the reference's Config, geoswe/solver.py:564-860).

The fields, defaults and validation follow the reference. This package runs the
production scheme only -- first-order SRM-HLLC, forward Euler, Sigma = 0 -- which is
what ``Config()`` selects; the research options the reference also accepts (LF
flux, higher-order reconstructions, SSP-RK3, IGR, Audusse) raise NotImplementedError
here instead of silently running another scheme.
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass
from typing import Optional

import numpy as np

G = 9.81
H_MIN = 1.0e-10

_BC_OK = {"extrapolate", "periodic", "wall", "fall", "dirichlet"}


def check_numeric_inputs(where="Config", **vals):
    """Bounds on the numeric inputs (geoswe/solver.py:564-626)."""
    def _f(name):
        v = vals.get(name, None)
        return None if v is None else float(v)

    for name, v in list(vals.items()):
        if v is not None and not math.isfinite(float(v)) and name != "friction_velocity_cap_ms":
            raise ValueError(f"{where}.{name}={v!r} is not finite")
    cfl = _f("cfl")
    if cfl is not None and not (0.0 < cfl <= 1.0):
        raise ValueError(f"{where}.cfl={cfl} is outside (0, 1]: the explicit step is unstable "
                         f"above the Courant limit. The published runs use 0.5.")
    if cfl is not None and cfl > 0.5:
        warnings.warn(f"{where}.cfl={cfl} is above 0.5; with the max(|u|,|v|) norm the 2D limit is "
                      f"near 0.5.", stacklevel=3)
    g = _f("g")
    if g is not None and g <= 0.0:
        raise ValueError(f"{where}.g={g} must be positive")
    h_min = _f("h_min")
    if h_min is not None and h_min <= 0.0:
        raise ValueError(f"{where}.h_min={h_min} must be positive (wet/dry threshold and divisor)")
    hmc = _f("h_min_cfl")
    if hmc is not None and hmc < 0.0:
        raise ValueError(f"{where}.h_min_cfl={hmc} must be >= 0 (0 couples it to h_min)")
    mn = _f("manning_n")
    if mn is not None and mn < 0.0:
        raise ValueError(f"{where}.manning_n={mn} must be >= 0")
    vcap = _f("friction_velocity_cap_ms")
    if vcap is not None and vcap <= 0.0:
        raise ValueError(f"{where}.friction_velocity_cap_ms={vcap} must be positive (inf disables)")
    rain = _f("rainfall")
    if rain is not None and rain > 1.0e-3:
        warnings.warn(f"{where}.rainfall={rain} is in m/s, not mm/h ({rain * 3.6e6:,.0f} mm/h).",
                      stacklevel=3)


@dataclass
class Config:
    """Solver configuration; ``Config()`` is the production flood scheme.

    Extensions over the reference: ``bc`` takes an optional per-face mapping
    ``{"x-": kind, "x+": kind, "y-": kind, "y+": kind}`` that overrides ``bc_x``/``bc_y``
    face by face (for example one open outflow edge on an otherwise walled domain).
    ``arith`` selects the step's arithmetic: ``"exact"`` (default; separately rounded
    IEEE operations and Manning's h^(-4/3) by CUDA's powf, as the reference kernel text:
    bit-identical to the reference kernel compiled without FMA contraction, friction
    included), ``"portable"`` (``"exact"`` with h^(-4/3) by a Newton iteration of IEEE
    operations, so a CPU reproduces every bit of a friction run; identical to
    ``"exact"`` without friction) or ``"fast"`` (binary32 only: FMA contraction,
    approximate square root and division; held to a depth tolerance against
    ``"exact"``, not to bit equality).
    """
    pde: str = "baseline"
    flux: str = "hllc"
    recon: str = "first"
    time: str = "euler"
    alpha: float = 0.0
    cfl: float = 0.5
    bc_x: str = "extrapolate"
    bc_y: str = "extrapolate"
    bc_x_left: Optional[np.ndarray] = None
    bc_x_right: Optional[np.ndarray] = None
    g: float = G
    h_min: float = H_MIN
    h_min_cfl: float = 0.0
    wb_method: str = "srm"
    friction: Optional[str] = None
    manning_n: float = 0.0
    friction_velocity_cap_ms: float = 15.0
    friction_quadratic_alpha: bool = True
    rainfall: float = 0.0
    rainfall_forcing: Optional[object] = None
    manning_field: Optional[np.ndarray] = None
    stage_boundary: Optional[object] = None
    well_balanced: bool = True
    dtype: Optional[str] = None
    wetdry_keep_h: bool = True
    bc: Optional[dict] = None
    arith: str = "exact"

    def __post_init__(self):
        if self.dtype is None:
            self.dtype = "float32"          # the GPU default, as in the reference on CuPy
        if not isinstance(self.dtype, str):
            try:
                self.dtype = np.dtype(self.dtype).name
            except TypeError:
                pass
        if self.dtype == "float32" and self.h_min == H_MIN:
            self.h_min = 1.0e-6
            if self.h_min_cfl == 0.0:
                self.h_min_cfl = self.h_min
        if isinstance(self.friction, str) and self.friction.lower() == "none":
            self.friction = None
        elif self.friction == "manning":
            self.friction = "manning_implicit"
        enum_ok = {"time": {"euler", "ssprk3"}, "flux": {"lf", "hllc"},
                   "recon": {"first", "muscl", "linear2", "linear3", "linear5", "weno5"},
                   "wb_method": {"audusse", "srm"}, "pde": {"igr", "baseline"},
                   "dtype": {"float32", "float64"}, "bc_x": _BC_OK, "bc_y": _BC_OK,
                   "friction": {"manning_implicit"}, "arith": {"exact", "fast", "portable"}}
        for k, ok in enum_ok.items():
            v = getattr(self, k, None)
            if v is None and k == "friction":
                continue
            if not isinstance(v, str) or v not in ok:
                raise ValueError(f"Config.{k}={v!r} invalid; expected one of {sorted(ok)}")
        if self.arith == "fast" and self.dtype != "float32":
            raise ValueError("Config.arith='fast' is binary32 only; use dtype='float32' or arith='exact'")
        if self.friction is None and (self.manning_n > 0.0 or self.manning_field is not None):
            warnings.warn("Config: a Manning roughness is set but friction is off, so the run is "
                          "frictionless; pass friction='manning' to apply it", stacklevel=3)
        check_numeric_inputs(where="Config", cfl=self.cfl, g=self.g, h_min=self.h_min,
                             h_min_cfl=self.h_min_cfl, manning_n=self.manning_n,
                             friction_velocity_cap_ms=self.friction_velocity_cap_ms,
                             rainfall=self.rainfall)
        if self.well_balanced and self.recon != "first":
            warnings.warn(f"Config.recon={self.recon!r} has no effect with well_balanced=True: the "
                          f"well-balanced face states are first order by construction.", stacklevel=3)
        if self.bc is not None:
            faces = {"x-", "x+", "y-", "y+"}
            bad = set(self.bc) - faces
            if bad:
                raise ValueError(f"Config.bc keys must be among {sorted(faces)}; got {sorted(bad)}")
            for f, kind in self.bc.items():
                if kind not in _BC_OK - {"dirichlet"}:
                    raise ValueError(f"Config.bc[{f!r}]={kind!r} invalid")

    # -- what this package runs ------------------------------------------------
    def require_production_scheme(self, who="Solver2D"):
        bad = []
        if self.flux != "hllc":
            bad.append(f"flux={self.flux!r}")
        if self.time != "euler":
            bad.append(f"time={self.time!r}")
        if not self.well_balanced or self.wb_method != "srm":
            bad.append("well_balanced=False" if not self.well_balanced else f"wb_method={self.wb_method!r}")
        if self.pde != "baseline" and self.alpha > 0.0:
            bad.append(f"pde={self.pde!r}")
        if bad:
            raise NotImplementedError(
                f"{who}: this package runs the production scheme (SRM-HLLC, forward Euler, "
                f"Sigma = 0); not supported: {', '.join(bad)}")

    def face_kinds(self):
        """Boundary kind per face (x-, x+, y-, y+)."""
        kinds = {"x-": self.bc_x, "x+": self.bc_x, "y-": self.bc_y, "y+": self.bc_y}
        if self.bc:
            kinds.update(self.bc)
        return [kinds[f] for f in ("x-", "x+", "y-", "y+")]
