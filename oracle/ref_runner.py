"""The reference's dense GPU solver loop on its own kernels -- TEST INFRASTRUCTURE ONLY.

Drives oracle/_ref/libref_{fma,strict}.so (the reference's kernel text compiled by
oracle/ref_build.py) the way the reference's Solver2D drives them on CuPy:
apply_bc_2d (geoswe/bc.py:50-172) -> 2-D fused step (rhs_cuda.py:2151-2192, launched
as solver.py:2283-2296) -> swap -> t += dt, with cfl_dt from lammax_fp32_lean and the
host fp64 arithmetic of solver.py:2569-2666 and the run loop of solver.py:2975-3027.
Uniform rain is given to the fused kernel as a constant frame, which the reference
itself checks equals the uniform-rain split path bit for bit.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"


def available(variant="fma"):
    return (REF / f"libref_{variant}.so").exists()


def _lib(variant):
    L = C.CDLL(str(REF / f"libref_{variant}.so"))
    for n in ("ref_fstep2d", "ref_rhs_f32", "ref_rhs_f64", "ref_lammax"):
        getattr(L, n).restype = C.c_int
    return L


def _p(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def ref_residual(q_pad, b_pad, dx, dy, g, h_min, variant="fma", mask=None):
    """Residual of the reference's 2-D SRM-HLLC kernel on a padded state (numpy in/out)."""
    import torch
    L = _lib(variant)
    dt = q_pad.dtype
    q = torch.from_numpy(np.ascontiguousarray(q_pad)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(b_pad, dtype=dt)).cuda()
    r = torch.zeros_like(q)
    m = torch.from_numpy(np.ascontiguousarray(mask if mask is not None else
                                              np.ones(q_pad.shape[1:], np.uint8))).cuda()
    sig = torch.zeros(1, dtype=q.dtype, device="cuda")
    nxp, nyp = q_pad.shape[1:]
    if dt == np.float32:
        rc = L.ref_rhs_f32(_p(q[0]), _p(q[1]), _p(q[2]), _p(b), _p(r[0]), _p(r[1]), _p(r[2]), nxp, nyp,
                           C.c_float(1.0 / dx), C.c_float(1.0 / dy), C.c_float(g), C.c_float(h_min),
                           _p(m), _p(sig), _stream())
    else:
        rc = L.ref_rhs_f64(_p(q[0]), _p(q[1]), _p(q[2]), _p(b), _p(r[0]), _p(r[1]), _p(r[2]), nxp, nyp,
                           C.c_double(1.0 / dx), C.c_double(1.0 / dy), C.c_double(g), C.c_double(h_min),
                           _p(m), _p(sig), _stream())
    assert rc == 0, rc
    torch.cuda.synchronize()
    return r.cpu().numpy()


class RefDenseGPU:
    """fp32 dense run of the reference GPU path (its fused 2-D step kernel)."""

    def __init__(self, q_pad, b_pad, ngh, dx, dy, *, kinds=("extrapolate",) * 4, g=9.81, h_min=1e-6,
                 h_min_cfl=0.0, cfl=0.5, ncls=None, ntab=None, friction=False, vcap=15.0, quad=True,
                 rain_rate=None, variant="fma"):
        import torch
        self.L = _lib(variant)
        self.q = torch.from_numpy(np.ascontiguousarray(q_pad, dtype=np.float32)).cuda()
        self.qn = self.q.clone()
        self.b = torch.from_numpy(np.ascontiguousarray(b_pad, dtype=np.float32)).cuda()
        self.ngh, self.dx, self.dy, self.g, self.h_min, self.cfl = ngh, dx, dy, g, h_min, cfl
        hc = h_min_cfl if h_min_cfl > 0.0 else h_min
        self.h_cfl = max(hc, 1.0e-6)
        self.kinds = list(kinds)
        self.nxp, self.nyp = q_pad.shape[1:]
        nx, ny = self.nxp - 2 * ngh, self.nyp - 2 * ngh
        self.friction = friction
        if ncls is None:
            # friction off: the fused kernel always applies its friction block, so give it
            # n = 0 (alpha = 1 exactly while |U| stays under the velocity cap)
            ncls, ntab = np.zeros((self.nxp, self.nyp), np.uint8), [0.0]
        self.ncls = torch.from_numpy(np.ascontiguousarray(ncls, np.uint8)).cuda()
        self.ntab = torch.from_numpy(np.asarray(ntab, np.float32)).cuda()
        self.vcap, self.quad = vcap, quad
        self.rain_rate = rain_rate
        self.rain = None if rain_rate is None else torch.full((nx, ny), float(np.float32(rain_rate)),
                                                              dtype=torch.float32, device="cuda")
        self.max_h = torch.zeros((self.nxp, self.nyp), dtype=torch.float32, device="cuda")
        self.bits = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.ghost = torch.zeros(nx * ny, dtype=torch.uint8, device="cuda")
        self.dmask = torch.zeros(1, dtype=torch.uint8, device="cuda")
        self.dsig = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.dfl = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.t = 0.0
        self.nsteps = 0

    def apply_bc(self):
        q, n = self.q, self.ngh
        for face, kind in zip(("x-", "x+", "y-", "y+"), self.kinds):
            ax = 1 if face[0] == "x" else 2
            lo = face[1] == "-"
            N = q.shape[ax]
            for k in range(n):
                g = k if lo else N - 1 - k
                if kind == "extrapolate":
                    s = n if lo else N - n - 1
                elif kind == "wall":
                    s = 2 * n - 1 - k if lo else N - 2 * n + k
                elif kind == "periodic":
                    s = N - 2 * n + k if lo else 2 * n - 1 - k
                else:
                    s = None
                dst = q[:, g, :] if ax == 1 else q[:, :, g]
                if kind == "fall":
                    dst.zero_()
                    continue
                src = q[:, s, :] if ax == 1 else q[:, :, s]
                dst.copy_(src)
                if kind == "wall":
                    dst[ax].neg_()

    def cfl_dt(self):
        nx, ny = self.nxp - 2 * self.ngh, self.nyp - 2 * self.ngh
        self.bits.zero_()
        rc = self.L.ref_lammax(_p(self.q[0]), _p(self.q[1]), _p(self.q[2]), nx, ny, self.nyp, self.ngh,
                               C.c_float(self.g), C.c_float(self.h_cfl), _p(self.bits), _p(self.ghost), _stream())
        assert rc == 0
        lam = float(self.bits.cpu().numpy().view(np.float32)[0])
        if not math.isfinite(lam):
            raise FloatingPointError("non-finite max wave speed")
        floor = (self.g * self.h_cfl) ** 0.5
        if lam < floor:
            lam = floor
        return self.cfl * min(self.dx, self.dy) / (lam + 1.0e-12)

    def rain_step_limit(self, dt):
        if self.rain_rate is None or self.rain_rate <= 0.0:
            return dt
        dmin = min(self.dx, self.dy)
        return min(dt, (self.cfl * dmin) ** (2.0 / 3.0) / (self.g * float(self.rain_rate)) ** (1.0 / 3.0))

    def step(self, dt):
        self.apply_bc()
        use_tab = 1 if self.ncls is not None else 0
        rc = self.L.ref_fstep2d(
            _p(self.q[0]), _p(self.q[1]), _p(self.q[2]), _p(self.b), _p(self.qn[0]), _p(self.qn[1]),
            _p(self.qn[2]), self.nxp, self.nyp, C.c_float(1.0 / self.dx), C.c_float(1.0 / self.dy),
            C.c_float(self.g), C.c_float(self.h_min), _p(self.rain if self.rain is not None else self.dfl),
            1 if self.rain is not None else 0, _p(self.ncls if self.ncls is not None else self.dmask),
            _p(self.ntab if self.ntab is not None else self.dfl), _p(self.dfl), use_tab, _p(self.max_h), 1,
            self.ngh, C.c_float(dt), C.c_float(self.vcap), int(self.quad), _p(self.dmask), _p(self.dsig),
            _stream())
        assert rc == 0, rc
        self.q, self.qn = self.qn, self.q
        self.t += dt
        self.nsteps += 1
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


_FORCING = {"infiltrate": 0, "sponge": 1, "ga_drain": 2, "ga": 3, "drain_tau": 4, "clamp": 5, "drain_cap": 6}


def ref_forcing(which, q, *, cls=None, t0=None, t1=None, t2=None, F=None, Fmax=None, inv_tau=None, act=None,
                idx=None, a0=None, a1=None, n=None, dt=0.0, h_min=1e-6, variant="fma"):
    """Apply one of the reference's flat-loop forcing kernels (captured text, compiled by
    oracle/ref_build.py) in place on CUDA tensors in canonical flat order: q is a list
    of three float32 tensors; the other arrays as the kernel takes them."""
    L = _lib(variant)
    L.ref_forcing.restype = C.c_int
    if n is None:
        n = int(q[0].numel()) if idx is None else int(idx.numel())
    rc = L.ref_forcing(_FORCING[which], _p(q[0]), _p(q[1]), _p(q[2]), _p(cls), _p(t0), _p(t1), _p(t2), _p(F),
                       _p(Fmax), _p(inv_tau), _p(act), _p(idx), _p(a0), _p(a1), C.c_int(n),
                       C.c_float(dt), C.c_float(h_min), _stream())
    if rc != 0:
        raise RuntimeError(f"ref_forcing({which}): CUDA error {rc}")


class RefFlatGPU:
    """fp32 compressed-mesh run of the reference GPU path: its flat fused step + CFL kernel
    (chained neighbour preamble, no sigma, L2 or Linf wave-speed norm) on the canonical
    tables, driven by the reference's flat loop (geoswe/compressed_solver.py:2133-2400):
    the first dt from the standalone flat lammax (cfl_dt, :721-748), every later dt from the
    lambda the fused step reduced over the new state (dt_from_lam, :713-719), dt =
    min(dt, t_end - t), the rain row by searchsorted(right) - 1 clamped, t += dt, while
    t < t_end - 1e-9; rain on a dry bed bounds dt by (cfl dx)^(2/3) / (g R_max)^(1/3)
    (:3426-3431). No forcings, ring or inlets (the loop's fused-CFL path, :2100-2103).

    Arrays are canonical-order NumPy: nbr (N, 4) int16 deltas, is_active (N,) uint8,
    q (3, N) float32, bed (N,) float32, n_cls (N,) uint8, n_tab; rain_table (nt, ncol)
    float32 in m/s with rain_times (nt,) and rain_lookup (N,) int32."""

    def __init__(self, nbr, is_active, q, bed, dx, *, n_cls, n_tab, g=9.81, h_min=1e-6, cfl=0.5, linf=False,
                 vcap=15.0, quad=True, rain_times=None, rain_table=None, rain_lookup=None, dt_max=None,
                 variant="fma"):
        import torch
        self.L = _lib(variant)
        self.L.ref_flat_fstep.restype = C.c_int
        self.L.ref_flat_lammax.restype = C.c_int
        dev = "cuda"
        self.N = int(np.asarray(is_active).shape[0])
        self.nbr = torch.from_numpy(np.ascontiguousarray(nbr, dtype=np.int16).reshape(-1)).to(dev)
        self.act = torch.from_numpy(np.ascontiguousarray(is_active, dtype=np.uint8)).to(dev)
        self.q = [torch.from_numpy(np.ascontiguousarray(q[c], dtype=np.float32)).to(dev) for c in range(3)]
        self.qn = [torch.zeros_like(self.q[0]) for _ in range(3)]
        self.b = torch.from_numpy(np.ascontiguousarray(bed, dtype=np.float32)).to(dev)
        self.ncls = torch.from_numpy(np.ascontiguousarray(n_cls, dtype=np.uint8)).to(dev)
        self.ntab = torch.from_numpy(np.asarray(n_tab, dtype=np.float32)).to(dev)
        self.max_h = torch.zeros(self.N, dtype=torch.float32, device=dev)
        self.bits = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ones1 = torch.ones(1, dtype=torch.float32, device=dev)
        self.dummy = torch.zeros(4, dtype=torch.float32, device=dev)
        self.dx, self.g, self.h_min, self.cfl, self.linf = float(dx), float(g), float(h_min), float(cfl), int(bool(linf))
        self.h_min_cfl = max(float(h_min), 1.0e-6)
        self.vcap, self.quad = float(vcap), int(bool(quad))
        self.rain_on = rain_table is not None
        self.dt_max = dt_max
        if self.rain_on:
            tab = np.ascontiguousarray(rain_table, dtype=np.float32)
            self.rain_t = np.asarray(rain_times, dtype=np.float64)
            self.rate = torch.from_numpy(tab).to(dev)
            self.lk = torch.from_numpy(np.ascontiguousarray(rain_lookup, dtype=np.int32)).to(dev)
            rmax = float(tab.max())
            if rmax > 0.0:
                lim = (self.cfl * self.dx) ** (2.0 / 3.0) / (self.g * rmax) ** (1.0 / 3.0)
                self.dt_max = lim if self.dt_max is None else min(self.dt_max, lim)
        self.t = 0.0
        self.nsteps = 0

    def _float_bits(self):
        return float(self.bits.cpu().numpy().view(np.float32)[0])

    def cfl_dt(self):
        self.bits.zero_()
        rc = self.L.ref_flat_lammax(self.linf, _p(self.q[0]), _p(self.q[1]), _p(self.q[2]), _p(self.act),
                                    C.c_int(self.N), C.c_float(self.g), C.c_float(self.h_min),
                                    C.c_float(self.h_min_cfl), _p(self.bits), _p(self.dummy), _stream())
        assert rc == 0, rc
        lam = self._float_bits()
        if not (lam == lam and lam < float("inf")):
            return 0.0
        return self.dt_from_lam(lam)

    def dt_from_lam(self, lam):
        floor = (self.g * self.h_min) ** 0.5
        if lam < floor:
            lam = floor
        dt = self.cfl * self.dx / (lam + 1e-12)
        return dt if self.dt_max is None else min(dt, self.dt_max)

    def run(self, t_end, max_steps=10 ** 9):
        steps = 0
        lam_next = None
        while self.t < t_end - 1e-9 and steps < max_steps:
            dtl = self.dt_from_lam(lam_next) if lam_next is not None else self.cfl_dt()
            if not (dtl > 0.0):
                raise FloatingPointError("non-finite max wave speed")
            dt = min(dtl, t_end - self.t)
            if self.rain_on:
                it = max(0, min(self.rate.shape[0] - 1, int(np.searchsorted(self.rain_t, self.t, "right") - 1)))
                row, lk = self.rate[it], self.lk
            else:
                row, lk = self.dummy, self.dummy
            self.bits.zero_()
            rc = self.L.ref_flat_fstep(
                self.linf, _p(self.q[0]), _p(self.q[1]), _p(self.q[2]), _p(self.b), _p(self.qn[0]), _p(self.qn[1]),
                _p(self.qn[2]), C.c_int(self.N), C.c_float(1.0 / self.dx), C.c_float(self.g), C.c_float(self.h_min),
                _p(self.nbr), _p(self.act), _p(row), _p(lk), int(self.rain_on), _p(self.ones1), _p(self.ncls),
                _p(self.ntab), _p(self.max_h), 1, C.c_float(dt), C.c_float(self.vcap), self.quad, _p(self.bits),
                C.c_float(self.h_min_cfl), _p(self.dummy), _stream())
            assert rc == 0, rc
            self.q, self.qn = self.qn, self.q
            lam_next = self._float_bits()
            self.t += dt
            self.nsteps += 1
            steps += 1
        return steps
