"""CPU oracle for the GeoSWE finite-volume step -- TEST INFRASTRUCTURE ONLY.

This package is the checker: tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py use it to compute what the GPU kernels must produce. The product
(geoswe_b200) never imports it.

  * liboracle.so (gsw_oracle.c): per-cell C restatement of the reference's fused
    SRM-HLLC kernel text, CFL reductions and ghost fills, fp32 and fp64.
  * OracleSolver2D: the reference's dense time loop (geoswe/solver.py:2569-3027)
    driving those kernels, with dt/t arithmetic in Python floats as the reference
    host loop does, plus the stage boundary (geoswe/forcing.py:315-377) and the
    discharge inflow (geoswe/bc.py:175-235) restated in NumPy.
  * numpy_ref: a NumPy restatement of the reference's CPU path (Solver2D with the
    NumPy backend), the reference CPU implementation timed as the CPU baseline.
"""
from __future__ import annotations

import bisect
import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRC = [HERE / "gsw_oracle.c", HERE / "gsw_oracle_body.h"]


def build(force=False):
    """Compile liboracle.so with gcc (no fused multiply-add, no fast-math, OpenMP)."""
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= p.stat().st_mtime for p in SRC):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
                    "-shared", "-o", str(tmp), str(HERE / "gsw_oracle.c"), "-lm"], check=True)
    tmp.replace(LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        for sfx in ("f32", "f64"):
            getattr(_lib, f"gswo_dense_step_{sfx}").restype = C.c_double
            getattr(_lib, f"gswo_dense_lammax_{sfx}").restype = C.c_double
        _lib.gswo_pow_m43_f32.restype = C.c_double
        _lib.gswo_pow_m43_f32.argtypes = [C.c_float]
        _lib.gswo_pow_m43_f64.restype = C.c_double
        _lib.gswo_pow_m43_f64.argtypes = [C.c_double]
    return _lib


def _sfx(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def _R(dtype):
    return C.c_float if np.dtype(dtype) == np.float32 else C.c_double


def _p(a):
    return C.c_void_p(0) if a is None else a.ctypes.data_as(C.c_void_p)


BC = {"extrapolate": 0, "wall": 1, "fall": 2, "periodic": 3, "none": 4}


def dense_rhs(q, b, dx, dy, g, h_min, mask=None):
    """Residual (3, nxp, nyp) of the padded state q on cells [2, n-3]^2."""
    dt = q.dtype
    q = np.ascontiguousarray(q)
    b = np.ascontiguousarray(b, dtype=dt)
    nxp, nyp = q.shape[1:]
    r = np.zeros_like(q)
    R = _R(dt)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    getattr(lib(), f"gswo_dense_rhs_{_sfx(dt)}")(
        _p(q[0]), _p(q[1]), _p(q[2]), _p(b), C.c_int(nxp), C.c_int(nyp), C.c_int64(nyp),
        R(1.0 / dx), R(1.0 / dy), R(g), R(h_min), _p(m), _p(r[0]), _p(r[1]), _p(r[2]))
    return r


def dense_step(q, b, ngh, dx, dy, g, h_min, dt, *, mask=None, rain=None, rain_kind=0,
               friction_kind=0, ncls=None, ntab=None, nfield=None, vcap=15.0, quad=True,
               keep_h=True, max_h=None, skip=None, h_cfl=None):
    """One fused step; returns (qn, lam_new)."""
    dtp = q.dtype
    q = np.ascontiguousarray(q)
    nxp, nyp = q.shape[1:]
    qn = np.empty_like(q)
    R = _R(dtp)
    conv = lambda a, d=dtp: None if a is None else np.ascontiguousarray(a, dtype=d)
    lam = getattr(lib(), f"gswo_dense_step_{_sfx(dtp)}")(
        _p(q[0]), _p(q[1]), _p(q[2]), _p(conv(b)), C.c_int(nxp), C.c_int(nyp), C.c_int(ngh),
        C.c_int64(nyp), R(1.0 / dx), R(1.0 / dy), R(g), R(h_min), R(dt),
        _p(conv(mask, np.uint8)), C.c_int(rain_kind), _p(conv(rain)), C.c_int(friction_kind),
        _p(conv(ncls, np.uint8)), _p(conv(ntab)), _p(conv(nfield)), R(vcap), C.c_int(int(quad)),
        C.c_int(int(keep_h)), _p(qn[0]), _p(qn[1]), _p(qn[2]), _p(max_h), _p(conv(skip, np.uint8)),
        R(h_cfl if h_cfl is not None else h_min))
    return qn, float(lam)


def dense_lammax(q, ngh, g, h_cfl, skip=None):
    dtp = q.dtype
    q = np.ascontiguousarray(q)
    nxp, nyp = q.shape[1:]
    R = _R(dtp)
    s = None if skip is None else np.ascontiguousarray(skip, dtype=np.uint8)
    return float(getattr(lib(), f"gswo_dense_lammax_{_sfx(dtp)}")(
        _p(q[0]), _p(q[1]), _p(q[2]), C.c_int(nxp), C.c_int(nyp), C.c_int(ngh), C.c_int64(nyp),
        R(g), R(h_cfl), _p(s)))


def bc_fill(q, ngh, kinds):
    """In-place ghost fill of the padded state (kinds for x-, x+, y-, y+)."""
    assert q.flags.c_contiguous
    nxp, nyp = q.shape[1:]
    k = (C.c_int * 4)(*[BC[x] for x in kinds])
    getattr(lib(), f"gswo_bc_{_sfx(q.dtype)}")(_p(q[0]), _p(q[1]), _p(q[2]), C.c_int(nxp),
                                                C.c_int(nyp), C.c_int(ngh), C.c_int64(nyp), k)


def pow_m43(x, dtype=np.float32):
    L = lib()
    return L.gswo_pow_m43_f32(float(x)) if np.dtype(dtype) == np.float32 else L.gswo_pow_m43_f64(float(x))


# ---------------------------------------------------------------------------
# Host-side pieces of the reference loop, restated.
# ---------------------------------------------------------------------------
def rain_index(time_s, t):
    """bisect_right(time_s, t) - 1, clamped (geoswe/forcing.py:191-193)."""
    tl = list(np.asarray(time_s, dtype=np.float64).tolist())
    idx = max(0, bisect.bisect_right(tl, float(t)) - 1)
    return min(idx, len(tl) - 1)


def stage_eta(time_s, stage_m, t):
    """Clamped linear interpolation (geoswe/forcing.py:283-313)."""
    tl = list(np.asarray(time_s, dtype=np.float64).tolist())
    sl = list(np.asarray(stage_m, dtype=np.float64).tolist())
    t = float(t)
    if t <= tl[0]:
        return sl[0]
    if t >= tl[-1]:
        return sl[-1]
    i = bisect.bisect_left(tl, t)
    w = (t - tl[i - 1]) / (tl[i] - tl[i - 1])
    return sl[i - 1] + w * (sl[i] - sl[i - 1])


def inflow_apply(q, bed, idx_i, idx_j, nx_n, ny_n, ds, Q, ngh, dry_frac=0.10):
    """Discharge inflow through the ghost cells (geoswe/bc.py:175-235), NumPy."""
    if len(idx_i) == 0:
        return
    h = q[0][idx_i, idx_j]
    z = bed[idx_i, idx_j]
    s = float(h.sum())
    if s > 0.0:
        w = h / s
        h_face = h
    else:
        zmin = z.min(); zmax = z.max()
        h_face = np.maximum(zmin + dry_frac * (zmax - zmin) - z, 0.0)
        low = (z <= zmin)
        n_low = float(low.sum())
        if float(h_face.max()) <= 0.0:
            q_cell = abs(Q) / (max(n_low, 1.0) * ds)
            h_face = h_face + (q_cell * q_cell / 9.80665) ** (1.0 / 3.0)
        w = np.where(low, 1.0 / max(n_low, 1.0), 0.0)
    qn = (Q / ds) * w
    si, sj = int(round(nx_n)), int(round(ny_n))
    for k in range(1, int(ngh) + 1):
        gi = idx_i - k * si
        gj = idx_j - k * sj
        q[0][gi, gj] = h_face
        q[1][gi, gj] = qn * nx_n
        q[2][gi, gj] = qn * ny_n


class OracleSolver2D:
    """The reference dense loop on the C oracle kernels (fp32 or fp64).

    Parameters mirror geoswe_b200.Solver2D: padded state (3, nxp, nyp) and bed, the
    face BC kinds, Manning (none / table / field / scalar), rain (none / uniform table /
    gridded frames with their times), stage boundaries and inflow inlets.
    """

    def __init__(self, q_pad, b_pad, ngh, dx, dy, *, g=9.81, h_min=1e-6, h_cfl=None, cfl=0.5,
                 kinds=("extrapolate",) * 4, mask=None, friction=None, ncls=None, ntab=None,
                 nfield=None, manning_n=0.0, vcap=15.0, quad=True, keep_h=True,
                 rain_times=None, rain_frames=None, rain_gridded=False, rain_rmax=None,
                 stages=(), inflows=(), ghost=None, track_max=True):
        self.q = np.ascontiguousarray(q_pad).copy()
        self.dtype = self.q.dtype
        self.b = np.ascontiguousarray(b_pad, dtype=self.dtype)
        self.ngh, self.dx, self.dy = ngh, dx, dy
        self.g, self.h_min, self.cfl = g, h_min, cfl
        hc = h_cfl if h_cfl is not None else h_min
        if self.dtype == np.float32 and hc < 1e-6:
            hc = 1e-6
        self.h_cfl = hc
        self.kinds = list(kinds)
        self.mask = mask
        self.vcap, self.quad, self.keep_h = vcap, quad, keep_h
        if friction is None:
            self.fk, self.ncls, self.ntab, self.nfield = 0, None, None, None
        elif ncls is not None:
            self.fk, self.ncls, self.ntab, self.nfield = 1, ncls, np.asarray(ntab, np.float32).astype(self.dtype), None
        elif nfield is not None:
            self.fk, self.ncls, self.ntab, self.nfield = 2, None, None, nfield
        else:   # scalar n: a one-entry table read for every cell
            self.fk = 1
            self.ncls = np.zeros(self.q.shape[1:], np.uint8)
            self.ntab = np.array([manning_n], dtype=self.dtype)
            self.nfield = None
        self.rain_times = None if rain_times is None else np.asarray(rain_times, np.float64)
        self.rain_frames = rain_frames
        self.rain_gridded = rain_gridded
        self.rain_rmax = rain_rmax
        self.stages = list(stages)
        self.inflows = list(inflows)
        nx, ny = self.q.shape[1] - 2 * ngh, self.q.shape[2] - 2 * ngh
        self.ghost = ghost
        skip = np.zeros((nx, ny), bool) if (ghost is not None or self.stages) else None
        if ghost is not None:
            skip |= ghost
        for s in self.stages:
            skip[np.asarray(s["cells"])[:, 0] - ngh, np.asarray(s["cells"])[:, 1] - ngh] = True
        self.skip = skip
        self.max_h = np.zeros(self.q.shape[1:], dtype=self.dtype) if track_max else None
        self.t = 0.0
        self.nsteps = 0
        self.dts = []

    def cfl_dt(self):
        lam = dense_lammax(self.q, self.ngh, self.g, self.h_cfl, self.ghost)
        if not math.isfinite(lam):
            raise FloatingPointError(f"non-finite max wave speed at t={self.t}")
        floor = (self.g * self.h_cfl) ** 0.5
        if lam < floor:
            lam = floor
        return self.cfl * min(self.dx, self.dy) / (lam + 1.0e-12)

    def _rain_now(self):
        if self.rain_times is None:
            return 0, None, 0.0
        k = rain_index(self.rain_times, self.t)
        return k, self.rain_frames[k], self.rain_rmax[k]

    def rain_step_limit(self, dt):
        if self.rain_times is None:
            return dt
        _, _, rmax = self._rain_now()
        if rmax <= 0.0:
            return dt
        dmin = min(self.dx, self.dy)
        return min(dt, (self.cfl * dmin) ** (2.0 / 3.0) / (self.g * rmax) ** (1.0 / 3.0))

    def step(self, dt):
        bc_fill(self.q, self.ngh, self.kinds)
        for f in self.inflows:
            Q = float(np.interp(self.t, f["t"], f["q"]))
            inflow_apply(self.q, self.b, f["i"], f["j"], f["nx"], f["ny"], f["ds"], Q, self.ngh,
                         f.get("dry_frac", 0.10))
        rk, rain = 0, None
        if self.rain_times is not None:
            _, frame, _ = self._rain_now()
            rk = 2 if self.rain_gridded else 1
            rain = np.asarray(frame, dtype=self.dtype).reshape(-1) if self.rain_gridded else \
                np.array([frame], dtype=self.dtype)
        qn, _ = dense_step(self.q, self.b, self.ngh, self.dx, self.dy, self.g, self.h_min,
                           self.dtype.type(dt), mask=self.mask, rain=rain, rain_kind=rk,
                           friction_kind=self.fk, ncls=self.ncls, ntab=self.ntab, nfield=self.nfield,
                           vcap=self.vcap, quad=self.quad, keep_h=self.keep_h, max_h=self.max_h,
                           skip=self.skip, h_cfl=self.h_cfl)
        self.q = qn
        self.t += dt
        for s in self.stages:
            eta = stage_eta(s["time_s"], s["stage_m"], self.t)
            bed = np.asarray(s["bed"])
            hn = np.maximum(eta - bed, 0.0)
            c = np.asarray(s["cells"])
            self.q[0][c[:, 0], c[:, 1]] = hn
            self.q[1][c[:, 0], c[:, 1]] = 0.0
            self.q[2][c[:, 0], c[:, 1]] = 0.0
        self.nsteps += 1
        self.dts.append(dt)
        return dt

    def run(self, t_end, max_steps=10 ** 7, dt_max=None):
        steps = 0
        while self.t < t_end - 1.0e-12 and steps < max_steps:
            dt = self.rain_step_limit(self.cfl_dt())
            if dt_max is not None and dt > dt_max:
                dt = dt_max
            if self.t + dt > t_end:
                dt = t_end - self.t
            self.step(dt)
            steps += 1
        return steps


# ---------------------------------------------------------------------------
# Compressed (flat) mesh: canonical order, int16 delta table (fp32).
# ---------------------------------------------------------------------------
def _flat_setup(L):
    for n in ("gswo_flat_step_f32", "gswo_flat_lammax_f32"):
        getattr(L, n).restype = C.c_double


def flat_rhs(nbr, act, q, b, dx, g, h_min):
    L = lib()
    N = len(act)
    q = [np.ascontiguousarray(x, np.float32) for x in q]
    r = [np.zeros(N, np.float32) for _ in range(3)]
    inv = C.c_float(np.float32(1.0 / dx))
    L.gswo_flat_rhs_f32(C.c_int64(N), _p(np.ascontiguousarray(nbr, np.int16)), _p(np.ascontiguousarray(act, np.uint8)),
                        _p(q[0]), _p(q[1]), _p(q[2]), _p(np.ascontiguousarray(b, np.float32)), inv, inv,
                        C.c_float(g), C.c_float(h_min), _p(r[0]), _p(r[1]), _p(r[2]))
    return np.stack(r)


class OracleFlat:
    """The reference's flat loop (geoswe/compressed_solver.py:713-748, 2133-2235) on the C
    oracle: canonical flat arrays, int16 neighbour deltas, the fused step's semantics."""

    def __init__(self, nbr, act, q, b, dx, *, g=9.81, h_min=1e-6, h_min_cfl=None, cfl=0.5, linf=False,
                 ncls=None, ntab=(0.0,), vcap=15.0, quad=True, keep_h=True, rain_times=None,
                 rain_table=None, rain_lookup=None, dt_max=None):
        L = lib()
        _flat_setup(L)
        self.L = L
        self.nbr = np.ascontiguousarray(nbr, np.int16)
        self.act = np.ascontiguousarray(act, np.uint8)
        self.q = [np.ascontiguousarray(x, np.float32).copy() for x in q]
        self.b = np.ascontiguousarray(b, np.float32)
        self.dx, self.g, self.cfl = dx, g, cfl
        self.h_min = max(h_min, 1e-6)
        self.h_min_cfl = max(self.h_min if h_min_cfl is None else h_min_cfl, 1e-6)
        self.linf = int(linf)
        self.ncls = None if ncls is None else np.ascontiguousarray(ncls, np.uint8)
        self.ntab = np.asarray(ntab, np.float32)
        self.vcap, self.quad, self.keep_h = vcap, quad, keep_h
        self.rain_times = None if rain_times is None else np.asarray(rain_times, np.float64)
        self.rain_table = None if rain_table is None else np.asarray(rain_table, np.float32)
        self.rain_lookup = rain_lookup
        self.dt_max = dt_max
        if self.rain_table is not None:
            rmax = float(self.rain_table.max())
            if rmax > 0.0:
                lim = (cfl * dx) ** (2.0 / 3.0) / (g * rmax) ** (1.0 / 3.0)
                self.dt_max = lim if self.dt_max is None else min(self.dt_max, lim)
        self.max_h = np.zeros(len(self.act), np.float32)
        self.t = 0.0
        self.nsteps = 0
        self._lam = None
        self.inflows = []

    def add_inflow(self, ghost_idx, nbr_idx, normal, ds, t_series, q_series):
        """A discharge inlet with the reference's dry seed (compressed_solver.py:1559-1594)."""
        a = np.asarray(nbr_idx, np.int64)
        zb = self.b[a]
        zmin, zmax = float(zb.min()), float(zb.max())
        h_dry = np.maximum(np.float32(zmin + 0.10 * (zmax - zmin)) - zb, np.float32(0.0))
        low = zb <= np.float32(zmin)
        nlow = float(low.sum()) or 1.0
        self.inflows.append(dict(g=np.asarray(ghost_idx, np.int64), a=a, nx=float(normal[0]),
                                 ny=float(normal[1]), ds=float(ds), t=np.asarray(t_series, np.float64),
                                 q=np.asarray(q_series, np.float64), h_dry=h_dry.astype(np.float32),
                                 nlow=nlow, flat=bool(float(h_dry.max()) <= 0.0),
                                 w_dry=np.where(low, np.float32(1.0 / nlow), np.float32(0.0))))
        return self

    def set_ring(self, ids, bed, wg, t_common, stage_all):
        """Ring stage on canonical ids (-1: skipped), as ring_bc_flat with the on-device
        interpolation (compressed_solver.py:287-307, 2338-2350)."""
        self.ring = dict(ids=np.asarray(ids, np.int64), bed=np.asarray(bed, np.float32),
                         wg=np.asarray(wg, np.float32).reshape(len(ids), -1),
                         t=np.asarray(t_common, np.float64), st=np.asarray(stage_all, np.float32))
        return self

    def set_forcings(self, *, infil_tab=None, sponge=None, ga=None, clamp=None, drain=None):
        """Per-step forcings on canonical ids, restated from the flat loop's kernels
        (compressed_solver.py:143-158, 268-283, 313-437, 1320-1328), applied in its order
        (:2330-2366): infiltration, sponge, ring, Green-Ampt / drain, clamp, drain cap.
        sponge = (ids, keep, amb); ga = dict(mode, cls, Ks, psi, dth, F, Fmax, inv_tau)
        (mode "ga" only: the drain's __expf has no exact CPU restatement); clamp = (ids,
        hmax); drain = (ids, h_tgt)."""
        self.forcings = dict(infil=infil_tab, sponge=sponge, ga=ga, clamp=clamp, drain=drain)
        return self

    def _apply_forcings(self, phase):
        f = getattr(self, "forcings", None)
        if not f:
            return
        q0, q1, q2 = self.q
        act = self.act != 0
        f32 = np.float32
        dt = f32(self._dt32)
        if phase == 0:
            if f["infil"] is not None:
                tab = np.asarray(f["infil"], np.float32)
                ncls = self.ncls if self.ncls is not None else np.zeros(len(self.act), np.uint8)
                m = act & (q0 >= f32(self.h_min))
                h = q0[m]
                hn = (h - (tab[ncls[m]] * dt).astype(np.float32)).astype(np.float32)
                hn = np.where(hn < 0, f32(0), hn).astype(np.float32)
                r = (hn / h).astype(np.float32)
                q0[m] = hn
                q1[m] = (q1[m] * r).astype(np.float32)
                q2[m] = (q2[m] * r).astype(np.float32)
            if f["sponge"] is not None:
                ids, keep, amb = f["sponge"]
                q0[ids] = ((q0[ids] * keep).astype(np.float32) + amb).astype(np.float32)
                q1[ids] = (q1[ids] * keep).astype(np.float32)
                q2[ids] = (q2[ids] * keep).astype(np.float32)
            return
        g = f["ga"]
        if g is not None:
            if g["mode"] != "ga":
                raise NotImplementedError("the oracle restates the Green-Ampt-only mode")
            K = np.asarray(g["Ks"], np.float32)[g["cls"]]
            m = act & (K > 0) & (q0 > 0)
            h = q0[m]
            KsDt = (K[m] * dt).astype(np.float32)
            head = (np.asarray(g["psi"], np.float32)[g["cls"][m]] + h).astype(np.float32)
            F0 = g["F"][m]
            A = (F0 + KsDt).astype(np.float32)
            disc = ((A * A).astype(np.float32)
                    + ((f32(4.0) * KsDt).astype(np.float32) * head).astype(np.float32)
                    * np.asarray(g["dth"], np.float32)[g["cls"][m]]).astype(np.float32)
            F1 = (f32(0.5) * (A + np.sqrt(np.maximum(disc, f32(0))).astype(np.float32)).astype(np.float32)
                  ).astype(np.float32)
            dF = np.maximum((F1 - F0).astype(np.float32), f32(0)).astype(np.float32)
            dF = np.where(dF > h, h, dF)
            Fmax = g["Fmax"][m] if g["Fmax"] is not None else np.full(h.size, f32(3.0e38), np.float32)
            room = (Fmax - F0).astype(np.float32)
            dF = np.where(dF > room, np.where(room > 0, room, f32(0)), dF).astype(np.float32)
            hn = (h - dF).astype(np.float32)
            al = (hn / h).astype(np.float32)
            q0[m] = hn
            q1[m] = (q1[m] * al).astype(np.float32)
            q2[m] = (q2[m] * al).astype(np.float32)
            g["F"][m] = (F0 + dF).astype(np.float32)
        for key, guard in (("clamp", False), ("drain", True)):
            if f[key] is None:
                continue
            ids, ht = f[key]
            for i, k in enumerate(ids):
                h = q0[k]
                if h > ht[i]:
                    r = (np.float32(ht[i] / h) if (not guard or h > np.float32(1e-12)) else np.float32(0.0))
                    q0[k] = ht[i]
                    q1[k] = np.float32(q1[k] * r)
                    q2[k] = np.float32(q2[k] * r)

    def _apply_ring(self):
        r = getattr(self, "ring", None)
        if r is None:
            return
        tc, st = r["t"], r["st"]
        ti = max(0, min(len(tc) - 2, int(np.searchsorted(tc, self.t) - 1)))
        wt = float((self.t - tc[ti]) / (tc[ti + 1] - tc[ti] + 1e-12))
        wt = min(1.0, max(0.0, wt))
        stage = (st[:, ti] * np.float32(1.0 - wt)).astype(np.float32)
        stage = (stage + st[:, ti + 1] * np.float32(wt)).astype(np.float32)
        eta = np.zeros(len(r["ids"]), np.float32)
        for g in range(stage.size):
            eta = (eta + r["wg"][:, g] * stage[g]).astype(np.float32)
        ok = r["ids"] >= 0
        idx = r["ids"][ok]
        self.q[0][idx] = np.maximum(np.float32(0.0), (eta - r["bed"])[ok]).astype(np.float32)
        self.q[1][idx] = np.float32(0.0)
        self.q[2][idx] = np.float32(0.0)

    def _apply_inflows(self):
        """The flat loop's inlet block (compressed_solver.py:2144-2167), NumPy sums."""
        q0, q1, q2 = self.q
        for f in self.inflows:
            Q = float(np.interp(self.t, f["t"], f["q"]))
            h_a = q0[f["a"]]
            ssum = float(h_a.sum())
            if ssum > 0.0:
                w = h_a / np.float32(ssum)
                h_face = h_a
            else:
                h_face = f["h_dry"]
                if f["flat"]:
                    qc = abs(Q) / (f["nlow"] * f["ds"])
                    h_face = h_face + np.float32((qc * qc / 9.80665) ** (1.0 / 3.0))
                w = f["w_dry"]
            qn = (np.float32(Q / f["ds"]) * w).astype(np.float32)
            q0[f["g"]] = np.asarray(h_face, np.float32)
            q1[f["g"]] = (qn * np.float32(f["nx"])).astype(np.float32)
            q2[f["g"]] = (qn * np.float32(f["ny"])).astype(np.float32)

    def _lammax(self):
        q = self.q
        return float(self.L.gswo_flat_lammax_f32(C.c_int64(len(self.act)), _p(self.act), _p(q[0]), _p(q[1]),
                                                 _p(q[2]), C.c_float(self.g), C.c_float(self.h_min),
                                                 C.c_float(self.h_min_cfl), C.c_int(self.linf)))

    def dt_from_lam(self, lam):
        floor = (self.g * self.h_min) ** 0.5
        if lam < floor:
            lam = floor
        dt = self.cfl * self.dx / (lam + 1e-12)
        return dt if self.dt_max is None else min(dt, self.dt_max)

    def step(self, dt):
        rate = None
        if self.rain_table is not None:
            it = max(0, min(self.rain_table.shape[0] - 1,
                            int(np.searchsorted(self.rain_times, self.t, "right") - 1)))
            rate = np.ascontiguousarray(self.rain_table[it][self.rain_lookup], np.float32)
        q = self.q
        qn = [np.empty_like(x) for x in q]
        inv = C.c_float(np.float32(1.0 / self.dx))
        lam = self.L.gswo_flat_step_f32(
            C.c_int64(len(self.act)), _p(self.nbr), _p(self.act), _p(q[0]), _p(q[1]), _p(q[2]), _p(self.b),
            inv, inv, C.c_float(self.g), C.c_float(self.h_min), C.c_float(self.h_min_cfl), C.c_int(self.linf),
            C.c_float(np.float32(dt)), _p(rate), _p(self.ncls), _p(self.ntab), C.c_float(self.vcap),
            C.c_int(int(self.quad)), C.c_int(int(self.keep_h)), _p(qn[0]), _p(qn[1]), _p(qn[2]), _p(self.max_h))
        self.q = qn
        self._lam = float(lam)
        self._dt32 = np.float32(dt)
        self._apply_forcings(0)
        self._apply_ring()                      # at the step's start time, after the step
        self._apply_forcings(1)
        if getattr(self, "forcings", None):
            self._lam = None                    # the wave speed of the forced state
        self.t += dt
        self.nsteps += 1

    def run(self, t_end, max_steps=10 ** 9):
        steps = 0
        while self.t < t_end - 1e-9 and steps < max_steps:
            lam = self._lammax() if self._lam is None else self._lam
            if not (lam == lam and lam < float("inf")):
                raise FloatingPointError("non-finite max wave speed")
            dt = min(self.dt_from_lam(lam), t_end - self.t)
            self._apply_inflows()
            self.step(dt)
            steps += 1
        return steps
