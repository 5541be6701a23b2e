"""Dense-grid solver: the reference's Solver2D (geoswe/solver.py:1273-3032) on libgsw.

The state lives on the GPU in two pitched buffers (ping-pong). One step is

    ghost fill -> inflow ghosts -> fused SRM-HLLC step -> t += dt -> stage boundary

exactly the order of Solver2D.step (solver.py:2695-2973), and `run` keeps dt, t, the
rain frame and the loop condition on the device (gsw_dt_finalize), capturing windows
of steps in CUDA graphs so the host only polls a done flag once per window.
"""
from __future__ import annotations

import ctypes as C
import math
import time
import warnings
from typing import Callable, Optional

import numpy as np
import torch

from . import _lib as L
from .config import Config
from .mesh import Mesh2D


def _pitch(n, itemsize):
    per = 128 // itemsize
    return ((n + per - 1) // per) * per


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("geoswe_b200 solvers run on a CUDA device (sm_100a); none is visible. "
                           "There is no CPU fallback; the CPU oracle under oracle/ is a test checker.")
    L.lib()


class _Tables:
    """Device copies of the forcing tables, in the solver's dtype."""


def _to_device(x, device, dtype):
    """A host array or tensor on `device` in `dtype`: one copy of the data as given
    (asynchronous from page-locked host memory), the dtype conversion on the device."""
    if not torch.is_tensor(x):
        x = torch.from_numpy(np.ascontiguousarray(x))
    pinned = x.device.type == "cpu" and x.is_pinned()
    return x.to(device, non_blocking=pinned).to(dtype)


def _loop_finished(st, p) -> bool:
    """True when the next evaluation of the dt rule (dt_finalize_one) would only commit the
    last step and stop the loop: the time has reached t_end - eps_end or the step count
    max_steps. The host then ends the loop itself (the caller commits the pending step)
    instead of launching one more window whose steps all find the loop done."""
    t_now = float(st.t_new) if st.pending else float(st.t)
    executed = int(st.steps) + int(st.pending)
    return not (t_now < p.t_end - p.eps_end) or (p.max_steps > 0 and executed >= p.max_steps)


def _cached_graph(cache, key, capture, device, keep=4):
    """The CUDA graph of `capture()` for `key`, captured on first use on a side stream
    (the captured kernels read the loop's `done` flag first, so a replay after the loop
    has finished is a no-op). At most `keep` graphs are kept."""
    if key not in cache:
        while len(cache) >= keep:
            cache.pop(next(iter(cache)))
        side = torch.cuda.Stream(device=device)
        side.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            per = capture()
        torch.cuda.current_stream().wait_stream(side)
        cache[key] = (g, per)
    return cache[key]


def pad_bed(bpad, ngh, bc_x, bc_y):
    """Ghost bed as the ghost state is filled (solver.py:1466-1484): x first over the
    full x extent, then y; a periodic axis wraps, every other kind repeats the edge
    cell. `bpad` is the padded (nxp, nyp) bed, a NumPy array or a tensor view, filled
    in place."""
    if bc_x == "periodic":
        bpad[:ngh, :] = bpad[-2 * ngh:-ngh, :]
        bpad[-ngh:, :] = bpad[ngh:2 * ngh, :]
    else:
        bpad[:ngh, :] = bpad[ngh:ngh + 1, :]
        bpad[-ngh:, :] = bpad[-ngh - 1:-ngh, :]
    if bc_y == "periodic":
        bpad[:, :ngh] = bpad[:, -2 * ngh:-ngh].clone() if torch.is_tensor(bpad) else bpad[:, -2 * ngh:-ngh]
        bpad[:, -ngh:] = bpad[:, ngh:2 * ngh].clone() if torch.is_tensor(bpad) else bpad[:, ngh:2 * ngh]
    else:
        bpad[:, :ngh] = bpad[:, ngh:ngh + 1]
        bpad[:, -ngh:] = bpad[:, -ngh - 1:-ngh]


class Solver2D:
    """Two-dimensional shallow-water solver on the dense padded grid.

    ``q0`` has shape (3, nx, ny) and ``b`` (nx, ny), host or device arrays. The padded
    state is exposed as ``q`` (a (3, nx+2ngh, ny+2ngh) CUDA tensor view) and the depth
    as ``depth()`` (NumPy). ``run``/``step``/``cfl_dt`` follow the reference.

    With ``comm`` (a torch.distributed process group of more than one rank) the run is
    split over the ranks of a ``dims`` Cartesian layout (solver.py:1286-1454): ``mesh``,
    ``q0`` and ``b`` are this rank's block (``partition.block_of``), faces that border
    another rank take their ghosts from it (``halo.Halo2D``; the bed once, the state
    every step) and the wave speed is the maximum over the ranks, so every rank takes
    the same dt and the blocks together equal the single-domain run bit for bit.
    """

    def __init__(self, mesh: Mesh2D, cfg: Config, q0, b, comm=None, dims=None, *,
                 device=None, track_max_depth: bool = True, use_graphs: bool = True,
                 tile_rows: int = 0, warps: int = 0, min_blocks: int = 0, autotuned: bool = True):
        _require_cuda()
        from .halo import comm_size
        self.comm = comm
        self.halo = None
        multi = comm_size(comm) > 1
        cfg.require_production_scheme("Solver2D")
        if "dirichlet" in (cfg.bc_x, cfg.bc_y):
            raise ValueError("bc 'dirichlet' exists for Solver1D only; in 2D impose a water "
                             "level with a StageBoundary (Config.stage_boundary)")
        self.mesh, self.cfg = mesh, cfg
        self.t = 0.0
        self.nsteps = 0
        self.diagnostics = {"rhs_calls": 0, "wallclock": 0.0}
        ngh = mesh.ngh
        if ngh < 2:
            raise ValueError(f"ngh={ngh} is too small: the fused SRM-HLLC step reads two cells "
                             f"beyond every interior cell. Construct Mesh2D with ngh >= 2.")
        if not torch.is_tensor(q0):
            q0 = np.asarray(q0)
        if not torch.is_tensor(b):
            b = np.asarray(b)
        if tuple(q0.shape) != (3, mesh.nx, mesh.ny):
            raise ValueError(f"q0 must have shape (3, nx, ny) = (3, {mesh.nx}, {mesh.ny}); "
                             f"got {tuple(q0.shape)}")
        if tuple(b.shape) != (mesh.nx, mesh.ny):
            raise ValueError(f"the bed must have shape (nx, ny) = ({mesh.nx}, {mesh.ny}); "
                             f"got {tuple(b.shape)}")
        rate = getattr(getattr(cfg, "rainfall_forcing", None), "rate_mm_h", None)
        if rate is not None and int(getattr(rate, "ndim", 1)) == 3 and tuple(rate.shape[1:]) != (mesh.nx, mesh.ny):
            raise ValueError(f"Config.rainfall_forcing.rate_mm_h has shape {tuple(rate.shape)}; gridded "
                             f"rain must be (nt, nx, ny) = (nt, {mesh.nx}, {mesh.ny})")
        if cfg.manning_field is not None:
            mf = np.asarray(cfg.manning_field.detach().cpu() if torch.is_tensor(cfg.manning_field)
                            else cfg.manning_field)
            if tuple(mf.shape) != mesh.padded_shape:
                raise ValueError(f"Config.manning_field must be the padded (nx+2*ngh, ny+2*ngh) = "
                                 f"{mesh.padded_shape} array, got {tuple(mf.shape)}")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.np_dtype = np.dtype(cfg.dtype)
        self.t_dtype = torch.float32 if self.np_dtype == np.float32 else torch.float64
        self.code = L.F32 if self.np_dtype == np.float32 else L.F64
        self.nxp, self.nyp = mesh.padded_shape
        self.pitch = _pitch(self.nyp, self.np_dtype.itemsize)
        self.arith = L.ARITH_CODES[cfg.arith]
        self._tile_rows, self._warps, self._min_blocks = int(tile_rows), int(warps), int(min_blocks)
        if autotuned and not (tile_rows or warps or min_blocks) and self.np_dtype == np.float32:
            from . import autotune
            best = autotune.load(autotune.kind("dense", self.arith), mesh.nx * mesh.ny)
            if best:
                self._tile_rows, self._warps = int(best["tile_rows"]), int(best["warps"])
                self._min_blocks = int(best["min_blocks"])
            elif mesh.nx * mesh.ny >= 1 << 20:
                self._min_blocks = 4     # untuned: the 64-register cap every large-grid tuning has chosen
        self._use_graphs = bool(use_graphs)
        dev, td = self.device, self.t_dtype
        self._buf = [torch.zeros((3, self.nxp, self.pitch), dtype=td, device=dev) for _ in range(2)]
        self._cur = 0
        # inputs go to the device as they are (one copy each, converted there); padding and
        # the finiteness check run on the device
        q_dev = _to_device(q0, dev, td)
        b_dev = _to_device(b, dev, td)
        fin_b, fin_q = torch.isfinite(b_dev).all(), torch.isfinite(q_dev).all()
        if not bool(fin_b & fin_q):          # one host synchronisation for both checks
            bad = "the bed" if not bool(fin_b) else "the initial state q0"
            raise ValueError(f"Solver2D: {bad} holds non-finite values (NaN or inf)")
        self._buf[0][:, ngh:ngh + mesh.nx, ngh:ngh + mesh.ny] = q_dev
        self._b = torch.zeros((self.nxp, self.pitch), dtype=td, device=dev)
        self._b[ngh:ngh + mesh.nx, ngh:ngh + mesh.ny] = b_dev
        self._pad_bed(self._b[:, :self.nyp])
        del q_dev, b_dev
        if multi:
            from .halo import Halo2D
            self.halo = Halo2D(comm, self.nxp, self.nyp, ngh, dtype=str(self.np_dtype),
                               periods=(cfg.bc_x == "periodic", cfg.bc_y == "periodic"),
                               dims=dims, device=self.device)
            # the bed's ghosts at a rank seam are the neighbour's cells, not the local
            # extrapolation (solver.py:1449-1454)
            self.halo.exchange(self._b)
            # the step sequence holds collectives; it is launched eagerly
            self._use_graphs = False
        self._mask = None
        self.inside_mask_interior = None
        self._ncls = None
        self._ntab = None
        self._nfield = None
        self._ghost = None             # interior cfl ghost mask (host bool)
        self._skip = None              # device uint8 (nx*ny): ghost | stage cells
        self._max_h = torch.zeros((self.nxp, self.pitch), dtype=td, device=dev) if track_max_depth else None
        self._stepped = False
        self._inflows = []
        self._state = torch.zeros(128, dtype=torch.uint8, device=dev)
        lam = L.GswLoopState.lam_bits.offset // 8
        self._lam_view = self._state.view(torch.int64)[lam:lam + 1]   # the wave-speed bits
        self._state_host = torch.zeros(128, dtype=torch.uint8).pin_memory()
        self._lam_scratch = torch.zeros(1, dtype=torch.int64, device=dev)
        self._graph_cache = {}
        self._dtp_dev = None
        self._dev_tables = None
        self._tables_key = None
        self.kernel_launches = 0        # libgsw kernels enqueued or replayed by this solver
        if cfg.manning_field is not None and cfg.friction is not None:
            self._nfield = torch.zeros((self.nxp, self.pitch), dtype=td, device=dev)
            self._nfield[:, :self.nyp].copy_(torch.from_numpy(np.ascontiguousarray(mf, dtype=self.np_dtype)))

    # ------------------------------------------------------------------ layout
    def _pad_bed(self, bpad):
        pad_bed(bpad, self.mesh.ngh, self.cfg.bc_x, self.cfg.bc_y)

    @property
    def q(self):
        """Padded conserved state (3, nxp, nyp): a CUDA tensor view of the current buffer."""
        return self._buf[self._cur][:, :, :self.nyp]

    @q.setter
    def q(self, value):
        v = value if torch.is_tensor(value) else torch.from_numpy(np.asarray(value))
        self._buf[self._cur][:, :, :self.nyp].copy_(v.to(self.t_dtype))
        self._invalidate()

    @property
    def b(self):
        return self._b[:, :self.nyp]

    @property
    def q_interior(self):
        g = self.mesh.ngh
        return self.q[:, g:-g, g:-g]

    def depth(self, out=None):
        """Water depth (nx, ny) as a NumPy array, ghost cells removed. ``out`` (an
        extension): a float (nx, ny) host array to copy into, e.g. page-locked memory,
        which is returned."""
        if out is None:
            return self.q_interior[0].detach().cpu().numpy()
        if tuple(out.shape) != (self.mesh.nx, self.mesh.ny):
            raise ValueError(f"depth(out=...): out must have shape ({self.mesh.nx}, {self.mesh.ny})")
        torch.from_numpy(out).copy_(self.q_interior[0].detach())
        return out

    def max_depth(self):
        """Running maximum depth after any step so far; depth() before the first step."""
        if self._max_h is None or not self._stepped:
            return self.depth()
        g = self.mesh.ngh
        return self._max_h[g:-g, g:self.nyp - g].detach().cpu().numpy()

    # ------------------------------------------------------------- set-up API
    def set_inside_mask(self, mask, cfl_robust_pct=None):
        """Active set (nx, ny) bool: cells outside get a zero residual and no rain."""
        if cfl_robust_pct is not None:
            raise NotImplementedError("cfl_robust_pct (a percentile dt limit) is not implemented; "
                                      "use set_cfl_ghost_mask to exclude cells from the dt limit")
        if mask is None:
            self._mask = None
            self.inside_mask_interior = None
            self._invalidate()
            return
        m = np.asarray(mask.detach().cpu() if torch.is_tensor(mask) else mask)
        if m.shape != (self.mesh.nx, self.mesh.ny):
            raise ValueError(f"inside_mask must have shape ({self.mesh.nx}, {self.mesh.ny}); got {m.shape}")
        ngh = self.mesh.ngh
        pad = np.zeros((self.nxp, self.pitch), dtype=np.uint8)
        pad[ngh:ngh + self.mesh.nx, ngh:ngh + self.mesh.ny] = m.astype(np.uint8)
        self._mask = torch.from_numpy(pad).to(self.device)
        self.inside_mask_interior = m.astype(bool)
        self._invalidate()

    @property
    def inside_mask(self):
        return None if self._mask is None else self._mask[:, :self.nyp]

    def set_manning_table(self, cls_padded, table):
        if not torch.is_tensor(cls_padded):
            cls_padded = torch.from_numpy(np.ascontiguousarray(cls_padded))
        table = np.asarray(table.detach().cpu() if torch.is_tensor(table) else table, dtype=np.float64)
        if tuple(cls_padded.shape) != (self.nxp, self.nyp):
            raise ValueError(f"set_manning_table expects a PADDED (nxp, nyp)={(self.nxp, self.nyp)} class "
                             f"array; got {tuple(cls_padded.shape)}")
        if cls_padded.dtype != torch.uint8:
            raise ValueError(f"set_manning_table: cls_padded must be uint8; got {cls_padded.dtype}")
        if table.ndim != 1 or table.size < 1 or table.size > 256:
            raise ValueError("set_manning_table: table must be 1-D with 1..256 entries")
        # one copy to the device (asynchronous from page-locked memory); checked and
        # pitched there
        pinned = cls_padded.device.type == "cpu" and cls_padded.is_pinned()
        cls_dev = cls_padded.to(self.device, non_blocking=pinned)
        cmax = int(cls_dev.max())
        if cmax >= int(table.size):
            raise ValueError(f"set_manning_table: class id {cmax} out of range for a "
                             f"{int(table.size)}-entry table")
        if self.cfg.friction is None:
            warnings.warn("set_manning_table: friction is off (Config.friction is None), so this "
                          "roughness table will not be applied", stacklevel=2)
        pad = torch.zeros((self.nxp, self.pitch), dtype=torch.uint8, device=self.device)
        pad[:, :self.nyp] = cls_dev
        self._ncls = pad
        self._ntab = torch.from_numpy(table.astype(np.float32).astype(self.np_dtype)).to(self.device)
        self._nfield = None
        self._invalidate()

    def set_manning(self, n):
        """Manning's n from a scalar or an (nx, ny) array; friction is switched on."""
        nx, ny, ngh = self.mesh.nx, self.mesh.ny, self.mesh.ngh
        n_host = np.asarray(n.detach().cpu() if torch.is_tensor(n) else n, dtype=np.float64)
        if n_host.ndim == 0:
            n_host = np.full((nx, ny), float(n_host))
        if n_host.shape != (nx, ny):
            raise ValueError(f"set_manning expects a scalar or an unpadded ({nx}, {ny}) array; got "
                             f"shape {n_host.shape}")
        if not np.all(np.isfinite(n_host)) or float(n_host.min()) < 0.0:
            raise ValueError("set_manning: Manning's n must be finite and non-negative")
        padded = np.pad(n_host, ngh, mode="edge")
        if self.cfg.friction is None:
            self.cfg.friction = "manning_implicit"
        self.cfg.manning_field = None
        vals, inv = np.unique(padded, return_inverse=True)
        if vals.size <= 256:
            self.set_manning_table(inv.reshape(padded.shape).astype(np.uint8), vals.astype(np.float32))
            return
        self._ncls = None
        self._ntab = None
        self._nfield = torch.zeros((self.nxp, self.pitch), dtype=self.t_dtype, device=self.device)
        self._nfield[:, :self.nyp].copy_(torch.from_numpy(padded.astype(self.np_dtype)))
        self._invalidate()

    def set_cfl_ghost_mask(self, mask):
        """Interior cells (nx, ny) excluded from the CFL wave speed."""
        if mask is None:
            self._ghost = None
        else:
            m = np.asarray(mask.detach().cpu() if torch.is_tensor(mask) else mask)
            if m.shape != (self.mesh.nx, self.mesh.ny):
                raise ValueError(f"cfl_ghost_mask must have shape ({self.mesh.nx}, {self.mesh.ny}); "
                                 f"got {m.shape}")
            self._ghost = m.astype(bool)
        self._invalidate()

    def add_inflow(self, idx_i, idx_j, normal, ds, t_series, q_series, dry_frac=0.10):
        """One discharge inlet on padded cells (idx_i, idx_j) along a physical edge;
        ``normal`` is the inward unit normal (axis-aligned)."""
        ii = np.asarray(idx_i, dtype=np.int64).ravel()
        jj = np.asarray(idx_j, dtype=np.int64).ravel()
        if ii.shape != jj.shape:
            raise ValueError("add_inflow: idx_i and idx_j must have the same length")
        si, sj = int(round(float(normal[0]))), int(round(float(normal[1])))
        if abs(si) + abs(sj) != 1:
            raise ValueError("add_inflow: the inward normal must be axis-aligned, one of (+-1, 0), (0, +-1)")
        ngh = self.mesh.ngh
        gi = ii[:, None] - np.arange(1, ngh + 1)[None, :] * si
        gj = jj[:, None] - np.arange(1, ngh + 1)[None, :] * sj
        if ii.size and (gi.min() < 0 or gi.max() >= self.nxp or gj.min() < 0 or gj.max() >= self.nyp):
            raise ValueError("add_inflow: the ghost cells outward of the inlet leave the padded grid")
        t = np.asarray(t_series, dtype=np.float64)
        qv = np.asarray(q_series, dtype=np.float64)
        if t.shape != qv.shape or t.ndim != 1 or t.size < 1:
            raise ValueError("add_inflow: t_series and q_series must be 1-D and of equal length")
        self._inflows.append(dict(i=ii, j=jj, nx=float(normal[0]), ny=float(normal[1]), ds=float(ds),
                                  t=t, q=qv, dry_frac=float(dry_frac), si=si, sj=sj))
        self._invalidate()

    def set_inflow(self, *a, **k):
        self._inflows = []
        self.add_inflow(*a, **k)

    def _invalidate(self):
        self._graph_cache.clear()
        self._dev_tables = None

    # --------------------------------------------------------------- tables
    def _h_cfl(self):
        cfg = self.cfg
        h = cfg.h_min_cfl if cfg.h_min_cfl > 0.0 else cfg.h_min
        if self.np_dtype == np.float32 and h < 1.0e-6:
            h = 1.0e-6
        return h

    def _stage_list(self):
        sb = self.cfg.stage_boundary
        if sb is None:
            return []
        return list(sb) if isinstance(sb, (list, tuple)) else [sb]

    def _tables(self):
        """Device tables for rain, stage, inflow and the CFL skip mask (built once)."""
        if self._dev_tables is not None:
            return self._dev_tables
        T = _Tables()
        dev, cfg = self.device, self.cfg
        nx, ny, ngh = self.mesh.nx, self.mesh.ny, self.mesh.ngh
        dmin = min(self.mesh.dx, self.mesh.dy)
        # rain (solver.py:1903-1914, forcing.py:170-216; rain limit solver.py:3005-3027)
        T.rain_kind = L.RAIN_NONE
        T.rain = T.rain_t = T.rain_lim = None
        rf = cfg.rainfall_forcing
        if rf is not None:
            frames = rf.frames(self.np_dtype)
            T.rain_kind = L.RAIN_GRIDDED if rf.gridded else L.RAIN_UNIFORM
            T.rain = torch.from_numpy(np.ascontiguousarray(frames)).to(dev)
            times = np.asarray(rf.time_s, dtype=np.float64)
            if rf.gridded:
                rmax = [float(frames[k].max()) for k in range(frames.shape[0])]
            else:
                rmax = [float(rf.rate_mm_h[k]) / 3.6e6 for k in range(len(times))]
        elif cfg.rainfall > 0.0:
            T.rain_kind = L.RAIN_UNIFORM
            T.rain = torch.tensor([cfg.rainfall], dtype=self.t_dtype, device=dev)
            times = np.array([0.0])
            rmax = [float(cfg.rainfall)]
        if T.rain_kind != L.RAIN_NONE:
            lim = [((cfg.cfl * dmin) ** (2.0 / 3.0) / (cfg.g * r) ** (1.0 / 3.0)) if r > 0.0 else 0.0
                   for r in rmax]
            T.rain_t = torch.from_numpy(times.copy()).to(dev)
            T.rain_lim = torch.tensor(lim, dtype=torch.float64, device=dev)
            T.n_rain = len(times)
        else:
            T.n_rain = 0
        # stage boundaries (forcing.py:315-377)
        T.stages = []
        skip = np.zeros((nx, ny), dtype=bool)
        if self._ghost is not None:
            skip |= self._ghost
        all_cells = []
        for sb in self._stage_list():
            cells = np.asarray(sb.cells, dtype=np.int64)
            if cells.size and (cells[:, 0].min() < ngh or cells[:, 0].max() >= ngh + nx or
                               cells[:, 1].min() < ngh or cells[:, 1].max() >= ngh + ny):
                raise ValueError("StageBoundary.cells must index the padded grid (unpadded index + "
                                 f"mesh.ngh = {ngh}); some cells lie in the ghost layers")
            off = cells[:, 0] * self.pitch + cells[:, 1]
            bed = np.asarray(sb.bed_b)
            d = dict(off=torch.from_numpy(off.astype(np.int64)).to(dev),
                     bed=torch.from_numpy(bed.astype(np.float64)).to(dev),
                     bed_f32=int(bed.dtype == np.float32), n=int(len(off)),
                     t=torch.from_numpy(np.asarray(sb.time_s, dtype=np.float64).copy()).to(dev),
                     s=torch.from_numpy(np.asarray(sb.stage_m, dtype=np.float64).copy()).to(dev),
                     nk=int(len(sb.time_s)))
            T.stages.append(d)
            skip[cells[:, 0] - ngh, cells[:, 1] - ngh] = True
            all_cells.append(cells)
        if all_cells:
            u = np.unique(np.concatenate(all_cells), axis=0)
            T.stage_union = torch.from_numpy((u[:, 0] * self.pitch + u[:, 1]).astype(np.int64)).to(dev)
            excl = np.zeros(len(u), dtype=np.uint8)
            if self._ghost is not None:
                excl = self._ghost[u[:, 0] - ngh, u[:, 1] - ngh].astype(np.uint8)
            T.stage_excl = torch.from_numpy(excl).to(dev)
        else:
            T.stage_union = None
        T.skip = torch.from_numpy(skip.astype(np.uint8).ravel()).to(dev) if skip.any() else None
        T.ghost_skip = (torch.from_numpy(self._ghost.astype(np.uint8).ravel()).to(dev)
                        if self._ghost is not None else None)
        # inflow inlets (solver.py:1916-1971)
        T.inflows = []
        for f in self._inflows:
            off = f["i"] * self.pitch + f["j"]
            T.inflows.append(dict(off=torch.from_numpy(off.astype(np.int64)).to(dev), n=int(len(off)),
                                  step=-(f["si"] * self.pitch + f["sj"]),
                                  t=torch.from_numpy(f["t"].copy()).to(dev),
                                  q=torch.from_numpy(f["q"].copy()).to(dev), nk=int(len(f["t"])), f=f))
        T.inlet_sums = None
        if self.halo is not None:
            # every rank posts one sum collective per step when there are inlets: the
            # counts must agree (a rank holding none of an inlet's cells lists it empty)
            self.halo.check_same(len(self._inflows), "Solver2D: discharge inlets")
            if self._inflows:
                T.inlet_sums = torch.zeros(len(self._inflows), dtype=torch.float64, device=dev)
        # friction
        if cfg.friction is None:
            T.fkind, T.ntab, T.ncls, T.nfield = L.FRICTION_NONE, None, None, None
        elif self._ncls is not None:
            T.fkind, T.ntab, T.ncls, T.nfield = L.FRICTION_TABLE, self._ntab, self._ncls, None
        elif self._nfield is not None:
            T.fkind, T.ntab, T.ncls, T.nfield = L.FRICTION_FIELD, None, None, self._nfield
        else:
            T.fkind, T.ncls, T.nfield = L.FRICTION_TABLE, None, None
            T.ntab = torch.tensor([float(self.np_dtype.type(cfg.manning_n))], dtype=self.t_dtype, device=dev)
        self._dev_tables = T
        return T

    # ---------------------------------------------------------- kernel calls
    def _dense_args(self, src, dst, T=None, step=True):
        cfg = self.cfg
        a = L.GswDenseArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = self.code
        a.nxp, a.nyp, a.ngh = self.nxp, self.nyp, self.mesh.ngh
        a.pitch = self.pitch
        a.q0, a.q1, a.q2 = _ptr(src[0]), _ptr(src[1]), _ptr(src[2])
        a.qn0, a.qn1, a.qn2 = _ptr(dst[0]), _ptr(dst[1]), _ptr(dst[2])
        a.bed = _ptr(self._b)
        a.inside_mask = _ptr(self._mask)
        a.mask_pitch = self.pitch
        a.inv_dx, a.inv_dy = 1.0 / self.mesh.dx, 1.0 / self.mesh.dy
        a.g, a.h_min = cfg.g, cfg.h_min
        a.h_cfl = self._h_cfl()
        a.tile_rows, a.warps, a.min_blocks = self._tile_rows, self._warps, self._min_blocks
        a.arith = self.arith
        if step:
            T = T or self._tables()
            a.state = _ptr(self._state)
            a.lam_target = C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset)
            a.rain_kind = T.rain_kind
            a.rain = _ptr(T.rain)
            a.friction_kind = T.fkind
            a.n_cls = _ptr(T.ncls)
            a.n_cls_pitch = self.pitch
            a.n_tab = _ptr(T.ntab)
            a.n_tab_len = int(T.ntab.numel()) if T.ntab is not None else 0
            a.n_field = _ptr(T.nfield)
            a.vcap = float(cfg.friction_velocity_cap_ms)
            a.quadratic = int(bool(cfg.friction_quadratic_alpha))
            a.keep_h = int(bool(cfg.wetdry_keep_h))
            a.max_h = _ptr(self._max_h)
            a.cfl_skip = _ptr(T.skip)
        return a

    def _bc_args(self, buf):
        a = L.GswBcArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = self.code
        a.nxp, a.nyp, a.ngh, a.pitch = self.nxp, self.nyp, self.mesh.ngh, self.pitch
        a.q0, a.q1, a.q2 = _ptr(buf[0]), _ptr(buf[1]), _ptr(buf[2])
        kinds = [L.BC_CODES[k] for k in self.cfg.face_kinds()]
        for f, side in enumerate(("x-", "x+", "y-", "y+")):
            # a face bordering another rank takes its ghosts from the halo exchange
            a.kinds[f] = L.BC_NONE if self.halo is not None and self.halo.has_neighbor(side) else kinds[f]
        a.state = _ptr(self._state)
        return a

    def _inflow_args(self, inl, src, hsum=None):
        f = inl["f"]
        a = L.GswInflowArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = self.code
        a.pitch = self.pitch
        a.q0, a.q1, a.q2 = _ptr(src[0]), _ptr(src[1]), _ptr(src[2])
        a.bed = _ptr(self._b)
        a.inlet_off = _ptr(inl["off"])
        a.n, a.ngh = inl["n"], self.mesh.ngh
        a.step_off = inl["step"]
        a.nx_n, a.ny_n, a.ds, a.dry_frac = f["nx"], f["ny"], f["ds"], f["dry_frac"]
        a.t_knots, a.q_knots, a.n_knots = _ptr(inl["t"]), _ptr(inl["q"]), inl["nk"]
        a.state = _ptr(self._state)
        a.hsum = hsum
        return a

    def _apply_inflows(self, T, src, s):
        """Inflow ghosts of every inlet on `src`; returns the kernels launched. On a split
        run an inlet may span ranks: each rank's depth sum, then one batched sum over the
        ranks for every inlet (solver.py:1956-1966), which the inflow kernels then use."""
        sums = [None] * len(T.inflows)
        n = len(T.inflows)
        if self.halo is not None and T.inflows:
            base = T.inlet_sums.data_ptr()
            sums = [C.c_void_p(base + 8 * k) for k in range(len(T.inflows))]
            for inl, p in zip(T.inflows, sums):
                L.call("gsw_inflow_depth_sum", C.byref(self._inflow_args(inl, src)), p, s)
            self.halo.allreduce_sum_(T.inlet_sums)
            n += len(T.inflows)
        for inl, p in zip(T.inflows, sums):
            L.call("gsw_inflow_apply", C.byref(self._inflow_args(inl, src, p)), s)
        return n

    def _launch_step(self, k_parity: int, T):
        """Ghost fill, inflow, fused step and stage for the buffer pair (k, 1-k)."""
        src, dst = self._buf[k_parity], self._buf[1 - k_parity]
        s = _stream()
        L.call("gsw_bc_fill", C.byref(self._bc_args(src)), s)
        n = 2 + 2 * len(T.stages) + (1 if len(T.stages) > 1 else 0)
        n += self._apply_inflows(T, src, s)
        windows = self._overlap_windows() if self.halo is not None else None
        if windows is None:
            if self.halo is not None:
                self.halo.exchange(src)
            L.call("gsw_dense_step", C.byref(self._dense_args(src, dst, T)), s)
        else:
            # the cells whose stencil reads no seam ghost step while the halo is in
            # flight; the bands next to the seams step once it has landed
            inner, bands = windows
            handle = self.halo.start_exchange(src)
            a = self._dense_args(src, dst, T)
            a.row_lo, a.row_hi, a.col_lo, a.col_hi = inner
            L.call("gsw_dense_step", C.byref(a), s)
            self.halo.wait_exchange(handle)
            for w in bands:
                a.row_lo, a.row_hi, a.col_lo, a.col_hi = w
                L.call("gsw_dense_step", C.byref(a), s)
            n += len(bands)
        self._counting += n
        multi = len(T.stages) > 1
        for st in T.stages:
            a = L.GswStageArgs()
            a.abi_version = L.ABI_VERSION
            a.dtype = self.code
            a.pitch = self.pitch
            a.q0, a.q1, a.q2 = _ptr(dst[0]), _ptr(dst[1]), _ptr(dst[2])
            a.cell_off, a.bed64, a.bed_is_f32, a.n_cells = _ptr(st["off"]), _ptr(st["bed"]), st["bed_f32"], st["n"]
            a.time_s, a.stage_m, a.n_knots = _ptr(st["t"]), _ptr(st["s"]), st["nk"]
            a.state = _ptr(self._state)
            a.g, a.h_cfl = self.cfg.g, self._h_cfl()
            if not multi:
                a.lam_target = C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset)
                a.cfl_ghost = _ptr(T.stage_excl)
            L.call("gsw_stage_apply", C.byref(a), s)
        if multi:   # fold the union of stage cells once, after every stage write
            a = L.GswStageArgs()
            a.abi_version = L.ABI_VERSION
            a.dtype = self.code
            a.pitch = self.pitch
            a.q0, a.q1, a.q2 = _ptr(dst[0]), _ptr(dst[1]), _ptr(dst[2])
            a.cell_off, a.n_cells = _ptr(T.stage_union), int(T.stage_union.numel())
            a.state = _ptr(self._state)
            a.lam_target = C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset)
            a.cfl_ghost = _ptr(T.stage_excl)
            a.g, a.h_cfl = self.cfg.g, self._h_cfl()
            L.call("gsw_lam_cells", C.byref(a), s)
        self.diagnostics["rhs_calls"] += 1

    _counting = 0

    def _overlap_windows(self):
        """(interior window, band windows) of a split run's step, as (row_lo, row_hi,
        col_lo, col_hi) of the padded grid: the interior leaves two rows (columns) next to
        every face that borders another rank -- the reach of the stencil -- and the bands
        are those rows (x seams, all columns) and columns (y seams, the interior rows).
        None when the block is too thin to leave an interior."""
        if getattr(self, "_windows_key", None) != (self.nxp, self.nyp):
            g, nxp, nyp, h = self.mesh.ngh, self.nxp, self.nyp, self.halo
            r0 = g + 2 if h.has_neighbor("x-") else g
            r1 = nxp - g - 2 if h.has_neighbor("x+") else nxp - g
            c0 = g + 2 if h.has_neighbor("y-") else g
            c1 = nyp - g - 2 if h.has_neighbor("y+") else nyp - g
            win = None
            if r1 > r0 and c1 > c0:
                bands = []
                if r0 > g:
                    bands.append((g, r0, g, nyp - g))
                if r1 < nxp - g:
                    bands.append((r1, nxp - g, g, nyp - g))
                if c0 > g:
                    bands.append((r0, r1, g, c0))
                if c1 < nyp - g:
                    bands.append((r0, r1, c1, nyp - g))
                win = ((r0, r1, c0, c1), bands)
            self._windows, self._windows_key = win, (self.nxp, self.nyp)
        return self._windows

    def _dt_params(self, t_end, dt_max=None, max_steps=0, fixed_dt=None):
        T = self._tables()
        cfg = self.cfg
        p = L.GswDtParams()
        p.abi_version = L.ABI_VERSION
        p.mode = 1 if fixed_dt is not None else 0
        p.cfl_dmin = cfg.cfl * min(self.mesh.dx, self.mesh.dy)
        p.lam_floor = (cfg.g * self._h_cfl()) ** 0.5
        p.t_end = float(t_end)
        p.eps_end = 1.0e-12
        p.dt_max = float(dt_max) if dt_max is not None else 0.0
        p.fixed_dt = float(fixed_dt) if fixed_dt is not None else 0.0
        p.max_steps = int(max_steps)
        if fixed_dt is None and T.n_rain:
            p.rain_t, p.rain_lim, p.n_rain = _ptr(T.rain_t), _ptr(T.rain_lim), T.n_rain
        elif T.n_rain:
            p.rain_t, p.rain_lim, p.n_rain = _ptr(T.rain_t), C.c_void_p(0), T.n_rain
        return p

    def _write_state(self, **kw):
        st = L.GswLoopState()
        st.t = float(kw.get("t", self.t))
        self._state_host.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))),
                                                dtype=torch.uint8))
        self._state.copy_(self._state_host, non_blocking=False)

    def _read_state(self) -> L.GswLoopState:
        self._state_host.copy_(self._state, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return L.GswLoopState.from_buffer_copy(bytes(self._state_host.numpy()[:C.sizeof(L.GswLoopState)]))

    def _lammax_into_state(self, skip):
        """Wave speed of the current state into state.lam_bits (the reference's cfl_dt pass)."""
        a = self._dense_args(self._buf[self._cur], self._buf[self._cur], step=False)
        a.cfl_skip = _ptr(skip)
        L.call("gsw_dense_lammax", C.byref(a),
               C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset), _stream())

    # --------------------------------------------------------------- public
    def apply_bc(self):
        """Fill the ghost cells of the current state: face kinds, then inflow ghosts at
        the current time (the reference's _apply_bc, solver.py:1750-1780)."""
        T = self._tables()
        self._write_state()
        src = self._buf[self._cur]
        s = _stream()
        L.call("gsw_bc_fill", C.byref(self._bc_args(src)), s)
        if self.halo is not None:
            self.halo.exchange(src)
        self._apply_inflows(T, src, s)

    def residual(self):
        """SRM-HLLC residual (3, nxp, nyp) of the current state on cells [2, n-3]^2, zero
        elsewhere and outside the inside mask -- the fused residual kernel of the
        reference (rhs_cuda.py:900-1207) without rain. Ghosts are used as they are;
        call apply_bc() first to refresh them."""
        out = torch.zeros((3, self.nxp, self.pitch), dtype=self.t_dtype, device=self.device)
        a = self._dense_args(self._buf[self._cur], out, step=False)
        L.call("gsw_dense_rhs", C.byref(a), _stream())
        return out[:, :, :self.nyp]

    def cfl_dt(self):
        """Global CFL time step (solver.py:2569-2693)."""
        T = self._tables()
        self._write_state()
        self._lammax_into_state(T.ghost_skip)
        if self.halo is not None:
            self.halo.allreduce_max_(self._lam_view)
        lam_max = self._read_state().lam_bits
        lam_max = float(np.array([lam_max], dtype=np.uint64).view(np.float64)[0])
        if not math.isfinite(lam_max):
            raise FloatingPointError(f"cfl_dt: non-finite max wave speed {lam_max} at t={self.t:.3f}s "
                                     f"-- NaN/Inf in hu/hv; check forcing/inputs")
        lam_floor = (self.cfg.g * self._h_cfl()) ** 0.5
        if lam_max < lam_floor:
            lam_max = lam_floor
        return self.cfg.cfl * min(self.mesh.dx, self.mesh.dy) / (lam_max + 1.0e-12)

    def step(self, dt: Optional[float] = None):
        """Advance one step of size dt (the CFL step when None); returns dt."""
        if dt is None:
            dt = self.cfl_dt()
        dt = float(dt)
        T = self._tables()
        self._write_state()
        p = self._dt_params(t_end=math.inf, fixed_dt=dt)
        s = _stream()
        self._counting = 0
        L.call("gsw_dt_finalize", C.byref(p), _ptr(self._state), s)
        self._launch_step(self._cur, T)
        L.call("gsw_loop_commit", _ptr(self._state), s)
        self.kernel_launches += self._counting + 2
        self._cur = 1 - self._cur
        self._stepped = True
        self.t += dt
        self.nsteps += 1
        self.last_dt = dt
        return dt

    def _rain_step_limit(self, dt):
        cfg = self.cfg
        if cfg.rainfall_forcing is not None:
            rate = cfg.rainfall_forcing.rate_at_time(self.t, self.np_dtype if cfg.rainfall_forcing.gridded else None)
        elif cfg.rainfall > 0.0:
            rate = cfg.rainfall
        else:
            return dt
        rmax = float(rate.max()) if getattr(rate, "ndim", 0) else float(rate)
        if rmax <= 0.0:
            return dt
        dmin = min(self.mesh.dx, self.mesh.dy)
        return min(dt, (cfg.cfl * dmin) ** (2.0 / 3.0) / (cfg.g * rmax) ** (1.0 / 3.0))

    def run(self, t_end: float, max_steps: int = 10 ** 7, callback: Optional[Callable] = None,
            dt_max: Optional[float] = None, window: int = 0):
        """Step to ``t_end`` with CFL steps (the rain film limit and ``dt_max`` applied,
        the last step clipped onto ``t_end``); returns the number of steps taken.

        Without a callback the loop runs on the device: dt, t and the rain frame are
        computed by gsw_dt_finalize and ``window`` steps at a time are replayed from a
        CUDA graph. With a callback each step returns to the host, as in the reference.
        """
        t0 = time.perf_counter()
        for sb in self._stage_list():
            sb.warn_if_uncovered(t_end)
        if callback is not None:
            steps = 0
            while self.t < t_end - 1.0e-12 and steps < max_steps:
                dt = self._rain_step_limit(self.cfl_dt())
                if dt_max is not None and dt > dt_max:
                    dt = dt_max
                if self.t + dt > t_end:
                    dt = t_end - self.t
                self.step(dt)
                steps += 1
                callback(self, steps)
            self.diagnostics["wallclock"] = time.perf_counter() - t0
            self.diagnostics["steps"] = steps
            return steps
        steps = self._run_device(t_end, max_steps, dt_max, window)
        self.diagnostics["wallclock"] = time.perf_counter() - t0
        self.diagnostics["steps"] = steps
        return steps

    def _window_size(self):
        n = self.mesh.nx * self.mesh.ny
        return 256 if n <= 1 << 20 else (64 if n <= 1 << 24 else 16)

    def _run_device(self, t_end, max_steps, dt_max, window=0):
        T = self._tables()
        K = int(window) if window else self._window_size()
        if self.halo is not None and not window:
            K = min(K, 32)     # launched eagerly: poll often, so few no-op steps follow the end
        use_graphs = self._use_graphs
        if max_steps and max_steps <= 2 * K and K <= 64 and not window:
            # a short run on a large grid: capturing a graph costs more than the few launches
            # it would save (each step is far longer than its launches), so launch eagerly
            use_graphs = False
            K = int(max_steps)
        elif max_steps and max_steps < K and not window:
            K = int(max_steps)
        K += K % 2
        self._write_state()
        self._lammax_into_state(T.ghost_skip)
        p = self._dt_params(t_end=t_end, dt_max=dt_max, max_steps=max_steps)
        # the dt rule is read from device memory, so one captured window serves every
        # t_end / dt_max / max_steps
        if self._dtp_dev is None:
            self._dtp_dev = torch.zeros(C.sizeof(L.GswDtParams), dtype=torch.uint8, device=self.device)
        L.call("gsw_dt_params_upload", C.byref(p), _ptr(self._dtp_dev), _stream())
        start_cur = self._cur

        def one_step(k_parity):
            if self.halo is not None:     # every rank takes the dt of the largest wave speed
                self.halo.allreduce_max_(self._lam_view)
            L.call("gsw_dt_finalize_dev", _ptr(self._dtp_dev), _ptr(self._state), _stream())
            self._counting += 1
            self._launch_step(k_parity, T)

        def one_window():
            self._counting = 0
            for k in range(K):
                one_step(k % 2)
            return self._counting

        lead = 0
        if start_cur == 1:
            # one step outside the window, so every captured window starts on buffer 0
            self._counting = 0
            one_step(1)
            lead = self._counting
        if use_graphs:
            g, per = _cached_graph(self._graph_cache, (K, self._tile_rows, self._warps, self._min_blocks),
                                   one_window, self.device)

            def run_window():
                g.replay()
                return per
        else:
            run_window = one_window
        self.kernel_launches += lead
        self.kernel_launches += 1            # the initial wave-speed pass
        while True:
            self.kernel_launches += run_window()
            st = self._read_state()
            if st.done or _loop_finished(st, p):
                break
        L.call("gsw_loop_commit", _ptr(self._state), _stream())
        self.kernel_launches += 1
        st = self._read_state()
        steps = int(st.steps)
        self._cur = (start_cur + steps) % 2
        if steps:
            self._stepped = True
            self.last_dt = float(st.dt)
        self.t = float(st.t)
        self.nsteps += steps
        if st.error == L.ERR_NONFINITE:
            raise FloatingPointError(f"cfl_dt: non-finite max wave speed {st.lam_used} at t={self.t:.3f}s "
                                     f"-- NaN/Inf in hu/hv; check forcing/inputs")
        return steps
