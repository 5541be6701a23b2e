"""Compressed active-cell mesh: the reference's CompressedSolver (geoswe/compressed_solver.py:
2882-3450) on libgsw.

Construction follows CompressedSolver.from_dense: the stored set is the inside mask of
the dense solver dilated twice with the 4-neighbour cross, the ring keeps the state it
had in the dense solver, and the scheme is fixed (first-order SRM-HLLC, forward Euler).
The reference's canonical flat tables (row-major ids, int16 E/W/N/S deltas, is_active)
are built bit-exactly on the host (gsw_mesh.cpp) and exposed as ``nbr``, ``is_active``
and ``ij_active``; the kernels run on a Hilbert-ordered brick layout of the same cells,
reached from the canonical order through ``slot_of`` (a permutation).
"""
from __future__ import annotations

import ctypes as C
import math
import time
import warnings
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .solver import Solver2D, _ptr, _stream

BRICK_W, BRICK_PITCH = L.BRICK_W, L.BRICK_PITCH
SLOT_STORED, SLOT_ACTIVE = 1, 2


GswFlatArgs = L.GswFlatArgs


def _host_lib():
    return L.lib()


def _check(rc):
    if rc != L.OK:
        raise L.GswError("mesh", rc, L.lib().gsw_last_error().decode(errors="replace"))


def build_tables(inside_pad: np.ndarray, ring: int = 2):
    """The reference's CompressedSWE tables for a padded inside mask (nxp, nyp):
    dict(N, N_active, ij (N,2) int32, nbr (N,4) int16, is_active (N) uint8,
    active_id (nxp, nyp) int32, fully_covered). Raises ValueError when a stored row is
    too wide for int16 deltas, as the reference does."""
    Lb = _host_lib()
    inside = np.ascontiguousarray(inside_pad, dtype=np.uint8)
    nxp, nyp = inside.shape
    ns, na = C.c_int64(), C.c_int64()
    _check(Lb.gsw_mesh_count(inside.ctypes.data, nxp, nyp, ring, C.byref(ns), C.byref(na)))
    N = ns.value
    ij = np.empty((N, 2), np.int32)
    nbr = np.empty((N, 4), np.int16)
    act = np.empty(N, np.uint8)
    aid = np.empty((nxp, nyp), np.int32)
    cov = C.c_int32()
    rc = Lb.gsw_mesh_build(inside.ctypes.data, nxp, nyp, ring, ij.ctypes.data, nbr.ctypes.data,
                           act.ctypes.data, aid.ctypes.data, C.byref(cov))
    if rc == L.ERR_RANGE:
        raise ValueError(Lb.gsw_last_error().decode())
    _check(rc)
    if not cov.value:
        warnings.warn("CompressedSWE: active set not fully covered by the stored ring -- affected "
                      "active cells fall back to a ghost stencil", stacklevel=2)
    return dict(N=N, N_active=na.value, ij=ij, nbr=nbr, is_active=act, active_id=aid,
                fully_covered=bool(cov.value))


def build_bricks(stored_pad: np.ndarray, brick_h: int):
    """Hilbert-ordered bricks of 30 x brick_h cells covering the stored cells."""
    Lb = _host_lib()
    st = np.ascontiguousarray(stored_pad, dtype=np.uint8)
    nxp, nyp = st.shape
    nb = C.c_int64()
    _check(Lb.gsw_bricks_build(st.ctypes.data, nxp, nyp, brick_h, C.byref(nb), None, None))
    bij = np.empty((nb.value, 2), np.int32)
    bnbr = np.empty((nb.value, 4), np.int32)
    _check(Lb.gsw_bricks_build(st.ctypes.data, nxp, nyp, brick_h, C.byref(nb), bij.ctypes.data,
                               bnbr.ctypes.data))
    return bij, bnbr


class CompressedSolver:
    """Shallow-water solver on the compressed active-cell mesh (GPU, float32)."""

    brick_h = 16

    @classmethod
    def from_dense(cls, s: Solver2D, *, cfl_linf: bool = False, dt_max=None, brick_h: Optional[int] = None,
                   track_max_depth: bool = True,
                   h_min: Optional[float] = None, cfl: Optional[float] = None, g: Optional[float] = None,
                   say=None):
        """Pack the dense solver ``s`` (its inside mask, state, bed, Manning) into the
        compressed layout. ``cfl_linf=True`` uses the dense solver's velocity norm in the
        time step."""
        cfg = s.cfg
        fixed = []
        if cfg.recon != "first":
            fixed.append(f"recon={cfg.recon!r}")
        if cfg.time != "euler":
            fixed.append(f"time={cfg.time!r}")
        if cfg.flux != "hllc":
            fixed.append(f"flux={cfg.flux!r}")
        if not cfg.well_balanced or cfg.wb_method != "srm":
            fixed.append("well_balanced/wb_method")
        if cfg.stage_boundary is not None:
            fixed.append("stage_boundary (not carried over)")
        if fixed:
            raise ValueError("CompressedSolver.from_dense: the compressed mesh runs first-order SRM-HLLC "
                             "with forward Euler; these Config choices cannot be honoured: " + "; ".join(fixed))
        if abs(float(s.mesh.dx) - float(s.mesh.dy)) > 1e-12:
            raise ValueError(f"CompressedSolver requires square cells; dense mesh has dx={s.mesh.dx} "
                             f"dy={s.mesh.dy}")
        if s.np_dtype != np.float32:
            raise ValueError("CompressedSolver runs in float32 (as the reference's compressed tier)")
        if cfg.bc_x != "fall" or cfg.bc_y != "fall":
            warnings.warn(f"CompressedSolver.from_dense: Config.bc_x={cfg.bc_x!r}, bc_y={cfg.bc_y!r} are not "
                          f"carried over. The compressed mesh closes its edge with the state stored in its "
                          f"ghost halo, which acts like the 'fall' boundary.", stacklevel=2)
        self = cls()
        self.brick_h = int(brick_h or cls.brick_h)
        self.device = s.device
        self.nxp, self.nyp, self.ngh = s.nxp, s.nyp, s.mesh.ngh
        self.nx, self.ny = s.mesh.nx, s.mesh.ny
        self.dx = float(s.mesh.dx)
        self.g = float(cfg.g if g is None else g)
        self.cfl = float(cfg.cfl if cfl is None else cfl)
        self.h_min = max(float(cfg.h_min), 1.0e-6) if h_min is None else float(h_min)
        self.h_min_cfl = max(self.h_min, 1.0e-6)
        self.cfl_linf = bool(cfl_linf)
        self.vcap = float(cfg.friction_velocity_cap_ms)
        self.quad = bool(cfg.friction_quadratic_alpha)
        self.keep_h = bool(cfg.wetdry_keep_h)
        self.dt_max_user = dt_max
        self._dense_had_rain = cfg.rainfall_forcing is not None or cfg.rainfall > 0.0
        t0 = time.perf_counter()
        dev = self.device
        g_ = s.mesh.ngh
        if s._mask is None:
            inside = torch.zeros((s.nxp, s.nyp), dtype=torch.uint8, device=dev)
            inside[g_:-g_, g_:-g_] = 1
        else:
            inside = s._mask[:, :s.nyp].contiguous()
        self._inside = inside
        # stored = inside dilated twice with the 4-neighbour cross (compressed_rhs.py:256)
        st = inside.bool()
        for _ in range(2):
            d = st.clone()
            d[1:, :] |= st[:-1, :]
            d[:-1, :] |= st[1:, :]
            d[:, 1:] |= st[:, :-1]
            d[:, :-1] |= st[:, 1:]
            st = d
        self._stored = st
        self.N_stored = int(st.sum())
        self.N_active = int(inside.sum())
        bij, bnbr = build_bricks(st.to(torch.uint8).cpu().numpy(), self.brick_h)
        self.n_bricks = int(len(bij))
        BS = self.brick_h * BRICK_PITCH
        self.nslots = (self.n_bricks + 1) * BS
        self._bij = torch.from_numpy(bij).to(dev)
        self._bnbr = torch.from_numpy(bnbr).to(dev)
        # slot -> padded (i, j) by arithmetic; canonical id = row-major rank among stored cells
        sl = torch.arange(self.n_bricks * BS, device=dev, dtype=torch.int64)
        b_ = sl // BS
        rem = sl - b_ * BS
        r_, c_ = rem // BRICK_PITCH, rem % BRICK_PITCH
        ii = self._bij[b_, 0].to(torch.int64) * self.brick_h + r_
        jj = self._bij[b_, 1].to(torch.int64) * BRICK_W + c_
        ok = (c_ < BRICK_W) & (ii < s.nxp) & (jj < s.nyp)
        ii, jj, sl = ii[ok], jj[ok], sl[ok]
        lin = ii * s.nyp + jj
        keep = st.reshape(-1)[lin]
        ii, jj, sl, lin = ii[keep], jj[keep], sl[keep], lin[keep]
        canon = torch.cumsum(st.reshape(-1).to(torch.int64), 0) - 1
        k = canon[lin]
        slot_of = torch.empty(self.N_stored, dtype=torch.int64, device=dev)
        slot_of[k] = sl
        self._slot = slot_of
        flags = torch.zeros(self.nslots, dtype=torch.uint8, device=dev)
        flags[sl] = (1 + 2 * inside.reshape(-1)[lin].to(torch.uint8))
        self._flags = flags
        pidx_of_slot = ii * s.pitch + jj

        def pack_dense(field2d_pitched, dtype=torch.float32):
            out = torch.zeros(self.nslots, dtype=dtype, device=dev)
            out[sl] = field2d_pitched.reshape(-1)[pidx_of_slot].to(dtype)
            return out

        self._tables_cache = None
        self._slot_cells = sl
        self._lin_of_slot = lin
        q = s._buf[s._cur]
        self._q = [[pack_dense(q[c]) for c in range(3)], [torch.zeros(self.nslots, device=dev) for _ in range(3)]]
        self._cur = 0
        self._b = pack_dense(s._b)
        T = s._tables()
        if T.fkind == L.FRICTION_TABLE and T.ncls is not None:
            self._ncls = pack_dense(T.ncls, torch.uint8)
            self._ntab = T.ntab.to(torch.float32).clone()
        elif T.fkind == L.FRICTION_FIELD:
            nf = T.nfield[:, :s.nyp].cpu().numpy()
            vals, inv = np.unique(nf, return_inverse=True)
            if vals.size > 256:
                raise ValueError("the compressed mesh stores Manning's n as a table of at most 256 classes")
            clsp = np.zeros((s.nxp, s.pitch), np.uint8)
            clsp[:, :s.nyp] = inv.reshape(nf.shape)
            self._ncls = pack_dense(torch.from_numpy(clsp).to(dev), torch.uint8)
            self._ntab = torch.from_numpy(vals.astype(np.float32)).to(dev)
        else:
            n = float(np.float32(cfg.manning_n)) if cfg.friction is not None else 0.0
            self._ncls = None
            self._ntab = torch.tensor([n], dtype=torch.float32, device=dev)
        self._max_h = torch.zeros(self.nslots, dtype=torch.float32, device=dev) if track_max_depth else None
        self._state = torch.zeros(128, dtype=torch.uint8, device=dev)
        self._state_host = torch.zeros(128, dtype=torch.uint8).pin_memory()
        self._rain = None
        self._rain_kind = L.RAIN_NONE
        self._rain_t = None
        self._rain_rmax = 0.0
        self._inflows = []
        self._ring = None
        self.warps, self.min_blocks = 0, 0
        from . import autotune
        best = autotune.load("flat", self.nslots)
        if best:
            self.warps, self.min_blocks = int(best["warps"]), int(best["min_blocks"])
        self._graph_cache = {}
        self.t = 0.0
        self.nsteps = 0
        self.kernel_launches = 0
        self.build_seconds = time.perf_counter() - t0
        if say:
            say(f"[compressed] N_active={self.N_active} N_stored={self.N_stored} bricks={self.n_bricks} "
                f"built in {self.build_seconds:.2f}s")
        return self

    # ------------------------------------------------------------- forcings
    def set_rain(self, rain):
        """Attach a RainfallForcing (uniform or (nt, nx, ny) gridded)."""
        if rain is None:
            self._rain, self._rain_kind, self._rain_t = None, L.RAIN_NONE, None
            return self
        rate = np.asarray(rain.rate_mm_h)
        t_s = np.asarray(rain.time_s, np.float64)
        if rate.ndim == 1:
            table = (np.asarray(rate, np.float64) / 3.6e6).astype(np.float32)
            self._rain_kind = L.RAIN_UNIFORM
        elif rate.ndim == 3 and tuple(rate.shape[1:]) == (self.nx, self.ny):
            table = (np.asarray(rate, np.float64).reshape(rate.shape[0], -1) / 3.6e6).astype(np.float32)
            self._rain_kind = L.RAIN_GRIDDED
        else:
            raise ValueError(f"set_rain: rate_mm_h must have shape (nt,) or (nt, {self.nx}, {self.ny}); "
                             f"got {tuple(rate.shape)}")
        self._rain = torch.from_numpy(np.ascontiguousarray(table)).to(self.device)
        self._rain_t = torch.from_numpy(t_s.copy()).to(self.device)
        self._rain_rmax = float(table.max())
        self._graph_cache.clear()
        return self

    def ghost_boundary_pairs(self):
        """Ghost (ring) cells that touch the active set, each with its first active
        neighbour in E, W, N, S order, as canonical flat indices (the pairing
        ``add_inflow`` takes; compressed_solver.py:468-483)."""
        nbr = self.nbr.astype(np.int64)
        act = self.is_active
        N = act.size
        k = np.arange(N, dtype=np.int64)
        best = np.full(N, -1, np.int64)
        ghost = act == 0
        for d in range(4):
            dl = nbr[:, d]
            cand = k + dl
            ok = (dl > -32768) & (cand >= 0) & (cand < N)
            cand = np.where(ok, cand, 0)
            ok &= (act[cand] != 0) & ghost & (best < 0)
            best = np.where(ok, cand, best)
        sel = best >= 0
        return k[sel], best[sel]

    def add_inflow(self, ghost_idx, nbr_idx, normal, ds, t_series, q_series):
        """Add one discharge (hydrograph) inlet (compressed_solver.py:3193-3207): ghost and
        active-neighbour cells as canonical flat indices (from ghost_boundary_pairs), the
        inward unit normal (axis-aligned), the cell width and the hydrograph Q(t) in m^3/s."""
        g = np.asarray(ghost_idx, np.int64).reshape(-1)
        a = np.asarray(nbr_idx, np.int64).reshape(-1)
        if g.size != a.size:
            raise ValueError("add_inflow: ghost_idx and nbr_idx must have the same length")
        nx_n, ny_n = (float(normal[0]), float(normal[1]))
        if sorted((abs(nx_n), abs(ny_n))) != [0.0, 1.0]:
            raise ValueError(f"add_inflow: the inward normal must be axis-aligned, got {normal}")
        t = np.asarray(t_series, np.float64).reshape(-1)
        qs = np.asarray(q_series, np.float64).reshape(-1)
        if t.size != qs.size or t.size < 1:
            raise ValueError("add_inflow: t_series and q_series must be non-empty and of equal length")
        if g.size:
            act = self.is_active
            if (g < 0).any() or (g >= act.size).any() or (a < 0).any() or (a >= act.size).any():
                raise ValueError("add_inflow: index out of range of the stored cells")
            if act[g].any() or not act[a].all():
                raise ValueError("add_inflow: ghost_idx must be ring cells and nbr_idx active cells")
        dev = self.device
        slot = self._slot
        self._inflows.append(dict(
            ghost=slot[torch.from_numpy(g).to(dev)].to(torch.int64).contiguous(),
            nbr=slot[torch.from_numpy(a).to(dev)].to(torch.int64).contiguous(),
            n=int(g.size), nx=nx_n, ny=ny_n, ds=float(ds),
            t=torch.from_numpy(t.copy()).to(dev), q=torch.from_numpy(qs.copy()).to(dev)))
        self._graph_cache.clear()
        return self

    def set_ring(self, ring):
        """Stage on ghost-ring cells (the reference's set_ring dict, compressed_solver.py:
        3146, 3264-3268, applied as ring_bc_flat after every step): keys i, j (padded
        indices of the ring cells), bed (their bed, float32), wg ((n, NG) gauge weights),
        NG, n, t_common (T times, s), stage_all ((NG, T) stages, m). None removes it."""
        if ring is None or int(ring.get("n", 0)) == 0:
            self._ring = None
            self._graph_cache.clear()
            return self
        n, NG = int(ring["n"]), int(ring["NG"])
        i = np.asarray(ring["i"], np.int64).reshape(-1)
        j = np.asarray(ring["j"], np.int64).reshape(-1)
        if i.size != n or j.size != n:
            raise ValueError("set_ring: i and j must hold n indices")
        t_c = np.asarray(ring["t_common"], np.float64).reshape(-1)
        st = np.asarray(ring["stage_all"], np.float32).reshape(NG, -1)
        if t_c.size < 2 or st.shape[1] != t_c.size:
            raise ValueError("set_ring: stage_all must be (NG, T) with T = len(t_common) >= 2")
        wg = np.asarray(ring["wg"], np.float32).reshape(n, NG)
        if (i < 0).any() or (i >= self.nxp).any() or (j < 0).any() or (j >= self.nyp).any():
            raise ValueError("set_ring: ring index outside the padded grid")
        dev = self.device
        lin = torch.from_numpy(i * self.nyp + j).to(dev)
        slot_of_cell = torch.full((self.nxp * self.nyp,), -1, dtype=torch.int64, device=dev)
        slot_of_cell[self._lin_of_slot.to(torch.int64)] = self._slot_cells.to(torch.int64)
        slots = slot_of_cell[lin].contiguous()
        del slot_of_cell
        self._ring = dict(slots=slots, n=n, NG=NG,
                          bed=torch.from_numpy(np.asarray(ring["bed"], np.float32).reshape(-1).copy()).to(dev),
                          wg=torch.from_numpy(wg.copy()).to(dev),
                          t=torch.from_numpy(t_c.copy()).to(dev),
                          stage=torch.from_numpy(np.ascontiguousarray(st)).to(dev))
        self._graph_cache.clear()
        return self

    def _ring_args(self, q):
        r = self._ring
        a = L.GswFlatRingArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = L.F32
        a.q0, a.q1, a.q2 = _ptr(q[0]), _ptr(q[1]), _ptr(q[2])
        a.slots, a.bed, a.wg = _ptr(r["slots"]), _ptr(r["bed"]), _ptr(r["wg"])
        a.n, a.NG = r["n"], r["NG"]
        a.t_common, a.n_t, a.stage_all = _ptr(r["t"]), int(r["t"].numel()), _ptr(r["stage"])
        a.state = _ptr(self._state)
        return a

    def _inflow_args(self, f, q):
        a = L.GswFlatInflowArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = L.F32
        a.q0, a.q1, a.q2, a.bed = _ptr(q[0]), _ptr(q[1]), _ptr(q[2]), _ptr(self._b)
        a.ghost_slot, a.nbr_slot, a.n = _ptr(f["ghost"]), _ptr(f["nbr"]), f["n"]
        a.nx_n, a.ny_n, a.ds = f["nx"], f["ny"], f["ds"]
        a.t_knots, a.q_knots, a.n_knots = _ptr(f["t"]), _ptr(f["q"]), int(f["t"].numel())
        a.state = _ptr(self._state)
        return a

    # ---------------------------------------------------------------- views
    def _canonical(self):
        """The reference's CompressedSWE tables of this mesh (host, bit-exact), built on
        first use: ij_active (N, 2), nbr (N, 4) int16 deltas, is_active (N)."""
        if self._tables_cache is None:
            self._tables_cache = build_tables(self._inside.cpu().numpy(), ring=2)
            assert self._tables_cache["N"] == self.N_stored
        return self._tables_cache

    @property
    def ij_active(self):
        return self._canonical()["ij"]

    @property
    def nbr(self):
        return self._canonical()["nbr"]

    @property
    def is_active(self):
        return self._canonical()["is_active"]

    @property
    def fully_covered(self):
        return self._canonical()["fully_covered"]

    @property
    def slot_of(self):
        return self._slot.cpu().numpy()

    @property
    def n_active(self):
        return int(self.N_active)

    @property
    def n_stored(self):
        return int(self.N_stored)

    def flat(self, c=0):
        """Field c of the current state in the reference's canonical flat order (N_stored,)."""
        return self._q[self._cur][c][self._slot]

    def depth(self):
        """Depth (nx, ny) as NumPy, zero outside the active set."""
        q = self._q[self._cur][0]
        out = torch.zeros(self.nxp * self.nyp, dtype=torch.float32, device=self.device)
        act = (self._flags & SLOT_ACTIVE) != 0
        out[self._lin_of_slot[act[self._slot_cells]]] = q[self._slot_cells][act[self._slot_cells]]
        g = self.ngh
        return out.reshape(self.nxp, self.nyp)[g:-g, g:-g].cpu().numpy()

    # ---------------------------------------------------------------- kernels
    def _args(self, src, dst, step=True):
        a = GswFlatArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = L.F32
        a.brick_h, a.n_bricks = self.brick_h, self.n_bricks
        a.brick_ij, a.brick_nbr, a.flags = _ptr(self._bij), _ptr(self._bnbr), _ptr(self._flags)
        a.q0, a.q1, a.q2 = _ptr(src[0]), _ptr(src[1]), _ptr(src[2])
        a.qn0, a.qn1, a.qn2 = _ptr(dst[0]), _ptr(dst[1]), _ptr(dst[2])
        a.bed = _ptr(self._b)
        inv = float(np.float32(1.0 / self.dx))
        a.inv_dx = a.inv_dy = inv
        a.g, a.h_min, a.h_min_cfl = self.g, self.h_min, self.h_min_cfl
        a.linf = int(self.cfl_linf)
        a.ngh, a.nx, a.ny = self.ngh, self.nx, self.ny
        a.warps, a.min_blocks = self.warps, self.min_blocks
        if step:
            a.state = _ptr(self._state)
            a.lam_target = C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset)
            a.rain_kind = self._rain_kind
            a.rain = _ptr(self._rain)
            a.n_cls, a.n_tab, a.n_tab_len = _ptr(self._ncls), _ptr(self._ntab), int(self._ntab.numel())
            a.vcap, a.quadratic, a.keep_h = self.vcap, int(self.quad), int(self.keep_h)
            a.max_h = _ptr(self._max_h)
        return a

    def residual(self):
        """Residual (3, N_stored) of the current state in canonical order (0 at ring cells)."""
        out = [torch.zeros(self.nslots, device=self.device) for _ in range(3)]
        a = self._args(self._q[self._cur], out, step=False)
        _host_lib()
        L.call("gsw_flat_rhs", C.byref(a), _stream())
        return torch.stack([o[self._slot] for o in out])

    def _write_state(self):
        st = L.GswLoopState()
        st.t = float(self.t)
        self._state_host.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))),
                                                dtype=torch.uint8))
        self._state.copy_(self._state_host)

    def _read_state(self):
        self._state_host.copy_(self._state, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return L.GswLoopState.from_buffer_copy(bytes(self._state_host.numpy()[:C.sizeof(L.GswLoopState)]))

    def _lammax_into_state(self):
        a = self._args(self._q[self._cur], self._q[self._cur], step=False)
        _host_lib()
        L.call("gsw_flat_lammax", C.byref(a),
               C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset), _stream())

    def _dt_params(self, t_end, dt_max, max_steps):
        p = L.GswDtParams()
        p.abi_version = L.ABI_VERSION
        p.mode = 0
        p.cfl_dmin = self.cfl * self.dx
        p.lam_floor = (self.g * self.h_min) ** 0.5
        p.t_end = float(t_end)
        p.eps_end = 1.0e-9
        dm = dt_max
        if self._rain_kind != L.RAIN_NONE and self._rain_rmax > 0.0:
            lim = (self.cfl * self.dx) ** (2.0 / 3.0) / (self.g * self._rain_rmax) ** (1.0 / 3.0)
            dm = lim if dm is None else min(dm, lim)
        p.dt_max = float(dm) if dm is not None else 0.0
        p.max_steps = int(max_steps)
        p.clip_flat = 1
        if self._rain_t is not None:
            p.rain_t, p.n_rain = _ptr(self._rain_t), int(self._rain_t.numel())
        return p

    def _window_size(self):
        n = self.N_stored
        return 256 if n <= 1 << 20 else (64 if n <= 1 << 24 else 16)

    def run(self, t_end=None, *, dt_max=None, max_steps: int = 10 ** 9, window: int = 0, say=None, **unused):
        """Step from the current time to ``t_end`` (the reference's flat loop,
        compressed_solver.py:2133-2448): dt from the previous step's wave speed, the rain
        film limit folded into dt_max, dt = min(dt, t_end - t). Returns the number of steps."""
        if t_end is None:
            raise TypeError("CompressedSolver.run() needs t_end, the end time in seconds")
        if self._rain is None and self._dense_had_rain:
            warnings.warn("CompressedSolver.run: the dense Config asked for rainfall and none was attached "
                          "here. from_dense does not carry rainfall over; pass the same RainfallForcing "
                          "to set_rain().", stacklevel=2)
        dm = dt_max if dt_max is not None else self.dt_max_user
        K = int(window) if window else self._window_size()
        if max_steps and max_steps < K:
            K = int(max_steps)
        K += K % 2
        self._write_state()
        self._lammax_into_state()
        p = self._dt_params(t_end, dm, max_steps)
        start = self._cur
        _host_lib()

        def one_window():
            s = _stream()
            for k in range(K):
                L.call("gsw_dt_finalize", C.byref(p), _ptr(self._state), s)
                src, dst = self._q[(start + k) % 2], self._q[(start + k + 1) % 2]
                for f in self._inflows:             # inlet ghosts at t_n, before the step
                    L.call("gsw_flat_inflow_apply", C.byref(self._inflow_args(f, src)), s)
                L.call("gsw_flat_step", C.byref(self._args(src, dst)), s)
                if self._ring is not None:          # ring stage at t_n, after the step
                    L.call("gsw_flat_ring_stage", C.byref(self._ring_args(dst)), s)
            return (2 + len(self._inflows) + (self._ring is not None)) * K

        key = (K, start, float(t_end), p.dt_max, int(max_steps), self._rain_kind, len(self._inflows),
               self._ring is not None, self.warps, self.min_blocks)
        if key not in self._graph_cache:
            self._graph_cache.clear()
            side = torch.cuda.Stream(device=self.device)
            side.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                per = one_window()
            torch.cuda.current_stream().wait_stream(side)
            self._graph_cache[key] = (g, per)
        g, per = self._graph_cache[key]
        self.kernel_launches += 1
        while True:
            g.replay()
            self.kernel_launches += per
            if self._read_state().done:
                break
        L.call("gsw_loop_commit", _ptr(self._state), _stream())
        self.kernel_launches += 1
        st = self._read_state()
        steps = int(st.steps)
        self._cur = (start + steps) % 2
        self.t = float(st.t)
        self.nsteps += steps
        if steps:
            self.last_dt = float(st.dt)
        if st.error == L.ERR_NONFINITE:
            raise FloatingPointError(f"cfl_dt: non-finite max wave speed at t={self.t:.3f}s "
                                     f"-- fp32 NaN/Inf in the state; check forcing/inputs")
        return steps
