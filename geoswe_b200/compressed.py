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
import time
import warnings
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .solver import Solver2D, _cached_graph, _loop_finished, _ptr, _stream

BRICK_W, BRICK_PITCH = L.BRICK_W, L.BRICK_PITCH
SLOT_STORED, SLOT_ACTIVE = 1, 2
# The order of a split cache's halo faces (CompressedHalo, compressed_solver.py:1127-1132)
HALO_FACE_ORDER = ("y-", "y+", "x-", "x+")


GswFlatArgs = L.GswFlatArgs


def _host_lib():
    return L.lib()


def _check(rc):
    if rc != L.OK:
        raise L.GswError("mesh", rc, L.lib().gsw_last_error().decode(errors="replace"))


# The reference's refusal of a mesh with no neighbour links at all (compressed_rhs.py:
# 222-224, nbr_to_int16_delta): no inside cell, or nothing stored around them.
_DEGENERATE = ("no interior neighbors (empty/degenerate active set) -- the inside mask selects no cell "
               "with a stored neighbour; check the mask and the ring width")


def build_tables(inside_pad: np.ndarray, ring: int = 2):
    """The reference's CompressedSWE tables for a padded inside mask (nxp, nyp):
    dict(N, N_active, ij (N,2) int32, nbr (N,4) int16, is_active (N) uint8,
    active_id (nxp, nyp) int32, fully_covered). Raises ValueError when a stored row is
    too wide for int16 deltas or when no cell has a stored neighbour, as the reference
    does."""
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
    if N == 0 or not (nbr != -32768).any():
        raise ValueError(_DEGENERATE)
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


def inlet_dry_reductions(zb, halo, device):
    """The dry-inlet seed's reductions over the ranks of a split run, as the reference
    makes them once (compressed_solver.py:1559-1594): for each inlet (zb[k], this rank's
    float32 bed values of its cells, possibly none), the bed minimum and maximum over
    every rank (one MIN all-reduce of (zmin, -zmax)), then the cells at that minimum (a
    SUM) and the largest seed depth max(seed - z, 0) with seed = float32(zmin + 0.10
    (zmax - zmin)) (a MAX). Returns one (zmin, zmax, nlow, hmax) per inlet; a rank
    without cells of an inlet contributes the neutral values."""
    n = len(zb)
    ext = torch.tensor([[float(z.min()), -float(z.max())] if z.size else [np.inf, np.inf] for z in zb],
                       dtype=torch.float64, device=device).reshape(n, 2)
    halo.allreduce_min_(ext)                              # NCCL reduces device tensors
    ext = ext.cpu()
    agg_n = torch.zeros(n, dtype=torch.float64)
    agg_h = torch.full((n,), -np.inf, dtype=torch.float64)
    for k, z in enumerate(zb):
        zmin, zmax = float(ext[k, 0]), -float(ext[k, 1])
        seed = np.float32(zmin + 0.10 * (zmax - zmin))        # the kernel's double arithmetic
        if z.size:
            agg_n[k] = float(np.count_nonzero(z <= np.float32(zmin)))
            agg_h[k] = float(np.maximum(seed - z, np.float32(0.0)).max())
    agg_n, agg_h = agg_n.to(device), agg_h.to(device)
    halo.allreduce_sum_(agg_n)
    halo.allreduce_max_(agg_h)
    agg_n, agg_h = agg_n.cpu(), agg_h.cpu()
    return [(float(ext[k, 0]), -float(ext[k, 1]), float(agg_n[k]), float(agg_h[k])) for k in range(n)]


class CompressedSolver:
    """Shallow-water solver on the compressed active-cell mesh (GPU, float32).

    Built by ``from_dense`` from a ``Solver2D`` split over ranks (``comm=``), it runs this
    rank's block: the neighbours' inside cells in the seam ghost rows are stored but not
    updated here, and before every step ``halo.FlatHalo`` refreshes them from the ranks
    that own them; the wave speed is the maximum over the ranks. The blocks equal the
    single-domain compressed run bit for bit (compressed_solver.py:1069-1310, 3079-3087).
    """

    brick_h = 16
    halo = None
    flat_halo = None

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
        self._init_physics(device=s.device, nxp=s.nxp, nyp=s.nyp, ngh=s.mesh.ngh, nx=s.mesh.nx, ny=s.mesh.ny,
                           dx=float(s.mesh.dx), g=float(cfg.g if g is None else g),
                           cfl=float(cfg.cfl if cfl is None else cfl),
                           h_min=max(float(cfg.h_min), 1.0e-6) if h_min is None else float(h_min),
                           cfl_linf=cfl_linf, vcap=float(cfg.friction_velocity_cap_ms),
                           quad=bool(cfg.friction_quadratic_alpha), keep_h=bool(cfg.wetdry_keep_h),
                           dt_max=dt_max, brick_h=brick_h, arith=cfg.arith)
        self._dense_had_rain = cfg.rainfall_forcing is not None or cfg.rainfall > 0.0
        t0 = time.perf_counter()
        dev = self.device
        g_ = s.mesh.ngh
        if s._mask is None:
            inside = torch.zeros((s.nxp, s.nyp), dtype=torch.uint8, device=dev)
            inside[g_:-g_, g_:-g_] = 1
        else:
            inside = s._mask[:, :s.nyp].contiguous()
        halo = getattr(s, "halo", None)
        if halo is None:
            sl, lin, ii, jj = self._build_layout(inside)
        else:
            if any(halo.periods):
                raise ValueError("CompressedSolver.from_dense: a split run with a periodic axis cannot be "
                                 "compressed (the compressed mesh has no periodic closure)")
            # the neighbours' inside cells in the seam ghost rows join the stored set's
            # seed, so every cell an active stencil here reads is stored on both ranks
            ext = inside.to(torch.float32)
            halo.exchange(ext)
            sl, lin, ii, jj = self._build_layout((ext > 0.5).to(torch.uint8), active=inside,
                                                 seams=[f for f in ("x-", "x+", "y-", "y+") if halo.has_neighbor(f)])
        pidx_of_slot = ii * s.pitch + jj

        def pack_dense(field2d_pitched, dtype=torch.float32):
            out = torch.zeros(self.nslots, dtype=dtype, device=dev)
            out[sl] = field2d_pitched.reshape(-1)[pidx_of_slot].to(dtype)
            return out

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
        self._init_runtime(track_max_depth)
        if halo is not None:
            from .halo import FlatHalo
            slot_pad = torch.full((s.nxp * s.nyp,), -1, dtype=torch.int64, device=dev)
            slot_pad[lin] = sl
            self.halo = halo
            self.flat_halo = FlatHalo(halo, slot_pad.reshape(s.nxp, s.nyp), nslots=self.nslots)
        self.build_seconds = time.perf_counter() - t0
        if say:
            say(f"[compressed] N_active={self.N_active} N_stored={self.N_stored} bricks={self.n_bricks} "
                f"built in {self.build_seconds:.2f}s")
        return self

    @classmethod
    def from_cache(cls, cache_dir, *, cfl: float = 0.5, h_min: float = 1e-6, g: float = 9.81, dt_max=None,
                   cfl_linf: bool = False, brick_h: Optional[int] = None, track_max_depth: bool = True,
                   device=None, say=None, arith: str = "exact", comm=None, dims=None):
        """Load a flat-mesh cache in the reference's format (save_cache /
        run_cached, compressed_solver.py:2504-2560, 2616-2780): meta.json plus .npy files
        (nbr int16 deltas, is_active, ij_active, q0..q2, bed_f, mcls_f, m_tab, and the
        ring and rain bundles), straight to the GPU without a dense domain. Physics
        scalars are the cached loop's (CFL, h_min, g as given; quadratic Manning, keep-h,
        15 m/s velocity cap). Porosity (Sigma), sponge and drain bundles are refused with
        an error.

        A cache of a run split over N ranks (one ``r##`` directory per rank, as the
        reference's save_cache writes under MPI) loads with ``comm`` (a process group of
        N ranks) and ``dims`` (the split, as for ``Solver2D``): each rank reads its own
        directory, keeps its stored cells and its active set as cached, and rebuilds the
        seam exchange, which is checked against the cached halo faces
        (compressed_solver.py:1127-1161, 2550-2557)."""
        import json
        import os
        t0 = time.perf_counter()
        rank, size = 0, 1
        if comm is not None:
            import torch.distributed as dist
            rank, size = dist.get_rank(comm), dist.get_world_size(comm)
        if size > 1:
            cache_dir = os.path.join(cache_dir, f"r{rank:02d}")
        path = lambda n: os.path.join(cache_dir, n)
        meta = json.load(open(path("meta.json")))
        split = bool(meta.get("mpi")) or int(meta.get("nranks", 1)) != 1
        if split != (size > 1) or int(meta.get("nranks", 1)) != size:
            raise ValueError(f"from_cache: the cache was written by {int(meta.get('nranks', 1))} rank(s); load it "
                             f"with comm= of as many ranks (got {size})")
        for key, what in (("has_sponge", "sponge"), ("has_drain", "drain")):
            if meta.get(key):
                raise NotImplementedError(f"from_cache: the cache holds a {what} bundle, which this solver "
                                          f"does not apply")
        ld = lambda n: np.load(path(n + ".npy"))
        nbr = ld("nbr")
        is_active = ld("is_active").astype(np.uint8)
        ij = ld("ij_active").astype(np.int64)
        N = int(is_active.shape[0])
        if int(meta.get("N", N)) != N or nbr.shape[0] != N or ij.shape[0] != N:
            raise RuntimeError(f"cache {cache_dir}: inconsistent row counts (torn or mixed-vintage cache)")
        if not bool(meta.get("no_sigma", True)) and os.path.exists(path("sig_f.npy")) and ld("sig_f").any():
            raise NotImplementedError("from_cache: porosity (Sigma) caches are not supported")
        nxp, nyp, ngh = int(meta["nxp"]), int(meta["nyp"]), int(meta["ngh"])
        self = cls()
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._init_physics(device=dev, nxp=nxp, nyp=nyp, ngh=ngh, nx=nxp - 2 * ngh, ny=nyp - 2 * ngh,
                           dx=float(meta["dx"]), g=g, cfl=cfl, h_min=max(float(h_min), 1.0e-6),
                           cfl_linf=cfl_linf, vcap=15.0, quad=True, keep_h=True, dt_max=dt_max, brick_h=brick_h,
                           arith=arith)
        self.cache_meta = meta
        inside = np.zeros((nxp, nyp), np.uint8)
        act = is_active != 0
        inside[ij[act, 0], ij[act, 1]] = 1
        halo = None
        if split:
            # the stored set is the cached one (own inside cells and the neighbours' in the
            # seam ghost rows, dilated); only the cached active cells are updated here
            from .halo import Halo2D
            halo = Halo2D(comm, nxp, nyp, ngh, dtype="float32", dims=dims)
            stored_mask = np.zeros((nxp, nyp), bool)
            stored_mask[ij[:, 0], ij[:, 1]] = True
            seams = [f for f in HALO_FACE_ORDER if halo.has_neighbor(f)]
            self._build_layout(torch.from_numpy(inside).to(dev), seams=seams,
                               stored=torch.from_numpy(stored_mask).to(dev))
            self._tables_cache = dict(ij=ij.astype(np.int32), nbr=nbr, is_active=is_active, N=N,
                                      fully_covered=None)
        else:
            self._build_layout(torch.from_numpy(inside).to(dev))
        stored = self._stored.cpu().numpy()
        canon_ij = np.argwhere(stored)
        if self.N_stored != N or not np.array_equal(canon_ij, ij):
            raise ValueError(f"cache {cache_dir}: its stored cells are not the two-cell ring of its active set "
                             f"in row-major order")
        slot = self._slot

        def pack(flat, dtype):
            out = torch.zeros(self.nslots, dtype=dtype, device=dev)
            out[slot] = torch.from_numpy(np.ascontiguousarray(flat)).to(dev).to(dtype)
            return out

        self._q = [[pack(ld(f"q{c}").astype(np.float32), torch.float32) for c in range(3)],
                   [torch.zeros(self.nslots, device=dev) for _ in range(3)]]
        self._cur = 0
        self._b = pack(ld("bed_f").astype(np.float32), torch.float32)
        self._ncls = pack(ld("mcls_f").astype(np.uint8), torch.uint8)
        self._ntab = torch.from_numpy(ld("m_tab").astype(np.float32).reshape(-1)).to(dev)
        self._init_runtime(track_max_depth)
        if meta.get("has_rain"):
            if os.path.exists(path("rain_lookup_flat.npz")):
                lookup = np.load(path("rain_lookup_flat.npz"))["lookup_flat"]
            else:
                lookup = ld("rain_lookup_flat")
            table = ld("rain_native_rate_dev").astype(np.float32)
            table = table.reshape(table.shape[0], -1)
            self._set_rain_table(np.asarray(ld("rain_t_s"), np.float64), table, pack(lookup.astype(np.int32),
                                                                                     torch.int32))
        if meta.get("has_ring"):
            rflat = ld("ring_rflat").astype(np.int64).reshape(-1)
            n, NG = int(meta["ring_n"]), int(meta["ring_NG"])
            if rflat.size and int(rflat.max()) >= N:
                raise RuntimeError(f"cache {cache_dir}: ring_rflat max >= N={N} (torn cache)")
            rf = torch.from_numpy(rflat).to(dev)
            slots = torch.where(rf >= 0, slot[rf.clamp_min(0)], torch.full_like(rf, -1))
            self._ring = dict(slots=slots.contiguous(), n=n, NG=NG,
                              bed=torch.from_numpy(ld("ring_rbed").astype(np.float32).reshape(-1)).to(dev),
                              wg=torch.from_numpy(ld("ring_rwg").astype(np.float32).reshape(n, NG)).to(dev),
                              t=torch.from_numpy(ld("ring_t_common").astype(np.float64).reshape(-1)).to(dev),
                              stage=torch.from_numpy(np.ascontiguousarray(
                                  ld("ring_stage_all").astype(np.float32).reshape(NG, -1))).to(dev))
        if split:
            from .halo import FlatHalo
            slot_pad = torch.full((nxp * nyp,), -1, dtype=torch.int64, device=dev)
            slot_pad[self._lin_of_slot] = self._slot_cells
            self.halo = halo
            self.flat_halo = FlatHalo(halo, slot_pad.reshape(nxp, nyp), nslots=self.nslots)
            faces = [s for s in HALO_FACE_ORDER if halo.has_neighbor(s)]
            cached = meta.get("halo_faces", [])
            if len(cached) != len(faces):
                raise RuntimeError(f"cache {cache_dir}: {len(cached)} halo faces cached, this split has {len(faces)}")
            for fi, (side, fm) in enumerate(zip(faces, cached)):
                n_send = np.load(path(f"halo_f{fi}_sfi.npy")).size
                n_recv = np.load(path(f"halo_f{fi}_rfi.npy")).size
                if (int(fm["nbr"]) != halo._neighbor(side) or n_send != self.flat_halo.send_cells(side)
                        or n_recv != int(self.flat_halo.faces[side]["rslot"].numel())):
                    raise RuntimeError(f"cache {cache_dir}: halo face {side} differs from this split's (neighbour "
                                       f"{fm['nbr']} vs {halo._neighbor(side)}, {n_send} vs "
                                       f"{self.flat_halo.send_cells(side)} cells sent); load with the dims it "
                                       f"was written with")
        self.build_seconds = time.perf_counter() - t0
        if say:
            say(f"[compressed] loaded {cache_dir}: N_active={self.N_active} N_stored={self.N_stored} "
                f"bricks={self.n_bricks} in {self.build_seconds:.2f}s")
        return self

    # ------------------------------------------------------------- construction
    def _init_physics(self, *, device, nxp, nyp, ngh, nx, ny, dx, g, cfl, h_min, cfl_linf, vcap, quad, keep_h,
                      dt_max, brick_h, arith="exact"):
        if arith not in L.ARITH_CODES:
            raise ValueError(f"CompressedSolver: arith={arith!r} invalid; expected one of {sorted(L.ARITH_CODES)}")
        self.arith = L.ARITH_CODES[arith]
        self.brick_h = int(brick_h or type(self).brick_h)
        self.device = torch.device(device)
        self.nxp, self.nyp, self.ngh = int(nxp), int(nyp), int(ngh)
        self.nx, self.ny = int(nx), int(ny)
        self.dx = float(dx)
        self.g, self.cfl, self.h_min = float(g), float(cfl), float(h_min)
        self.h_min_cfl = max(self.h_min, 1.0e-6)
        self.cfl_linf = bool(cfl_linf)
        self.vcap, self.quad, self.keep_h = float(vcap), bool(quad), bool(keep_h)
        self.dt_max_user = dt_max
        self._dense_had_rain = False

    def _build_layout(self, inside, active=None, seams=(), stored=None):
        """Stored set (the inside mask dilated twice with the 4-neighbour cross,
        compressed_rhs.py:256), Hilbert bricks, the canonical id -> slot map and the slot
        flags. `inside` is a device uint8 (nxp, nyp) mask; `active` (default `inside`)
        marks the cells this solver updates -- on a split run `inside` also holds the
        neighbours' inside cells in the seam ghost rows, stored but not updated here.
        `seams` names the faces ("x-", "x+", "y-", "y+") whose ghost strips another rank
        refreshes: the bricks that read a cell of those strips are moved to the end of
        the brick order (Hilbert order kept within each part), and `n_bricks_inner`
        counts the others, which the step updates while the seam exchange is in flight.
        `stored` (a device bool (nxp, nyp) mask) gives the stored set directly (a cache
        of a split run), instead of the dilation of `inside`.
        Returns (slots, padded linear index, i, j) of every stored cell."""
        dev = self.device
        self._inside = inside
        if active is None:
            active = inside
        st = inside.bool()
        for _ in range(2 if stored is None else 0):
            d = st.clone()
            d[1:, :] |= st[:-1, :]
            d[:-1, :] |= st[1:, :]
            d[:, 1:] |= st[:, :-1]
            d[:, :-1] |= st[:, 1:]
            st = d
        if stored is not None:
            st = stored.bool()
        self._stored = st
        self.N_stored = int(st.sum())
        self.N_active = int(active.sum())
        if self.N_stored == 0:
            raise ValueError(_DEGENERATE)
        bij, bnbr = build_bricks(st.to(torch.uint8).cpu().numpy(), self.brick_h)
        self.n_bricks = int(len(bij))
        self.n_bricks_inner = self.n_bricks
        if seams:
            bij, bnbr = self._seam_bricks_last(bij, bnbr, seams)
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
        ok = (c_ < BRICK_W) & (ii < self.nxp) & (jj < self.nyp)
        ii, jj, sl = ii[ok], jj[ok], sl[ok]
        lin = ii * self.nyp + jj
        keep = st.reshape(-1)[lin]
        ii, jj, sl, lin = ii[keep], jj[keep], sl[keep], lin[keep]
        canon = torch.cumsum(st.reshape(-1).to(torch.int64), 0) - 1
        k = canon[lin]
        slot_of = torch.empty(self.N_stored, dtype=torch.int64, device=dev)
        slot_of[k] = sl
        self._slot = slot_of
        flags = torch.zeros(self.nslots, dtype=torch.uint8, device=dev)
        flags[sl] = (1 + 2 * active.reshape(-1)[lin].to(torch.uint8))
        self._flags = flags
        self._tables_cache = None
        self._slot_cells = sl
        self._lin_of_slot = lin
        return sl, lin, ii, jj

    def _seam_bricks_last(self, bij, bnbr, seams):
        """Stable reorder of the bricks: those with a cell within 3 cells (rows or
        columns) of a seam ghost strip last. A brick's step reads its own cells and at
        most 2 rows and 2 columns beyond them (the x-face gradients' bed two rows out,
        the edge lanes' y-gradients one column beyond the neighbour brick's edge), so
        the bricks kept first read no seam ghost cell, and the copy of unchanged stored
        cells into the new state (seam ghosts included) is made by the bricks moved last."""
        g, reach, bh = self.ngh, 3, self.brick_h
        r0 = bij[:, 0].astype(np.int64) * bh
        c0 = bij[:, 1].astype(np.int64) * BRICK_W
        late = np.zeros(len(bij), bool)
        if "x-" in seams:
            late |= r0 < g + reach
        if "x+" in seams:
            late |= r0 + bh - 1 >= self.nxp - g - reach
        if "y-" in seams:
            late |= c0 < g + reach
        if "y+" in seams:
            late |= c0 + BRICK_W - 1 >= self.nyp - g - reach
        nb = len(bij)
        order = np.concatenate([np.nonzero(~late)[0], np.nonzero(late)[0]])
        new_of_old = np.empty(nb + 1, np.int64)
        new_of_old[order] = np.arange(nb)
        new_of_old[nb] = nb                                  # the all-zero brick stays last
        self.n_bricks_inner = int((~late).sum())
        return (np.ascontiguousarray(bij[order]),
                np.ascontiguousarray(new_of_old[bnbr[order].astype(np.int64)].astype(np.int32)))

    def _init_runtime(self, track_max_depth):
        dev = self.device
        self._max_h = torch.zeros(self.nslots, dtype=torch.float32, device=dev) if track_max_depth else None
        self._state = torch.zeros(128, dtype=torch.uint8, device=dev)
        self._state_host = torch.zeros(128, dtype=torch.uint8).pin_memory()
        self._rain = None
        self._rain_kind = L.RAIN_NONE
        self._rain_t = None
        self._rain_rmax = 0.0
        self._rain_lookup = None
        self._rain_ncol = 0
        self._inflows = []
        self._ring = None
        self._forcing = {}
        self.warps, self.min_blocks, self.segments = 0, 0, 0
        from . import autotune
        best = autotune.load(autotune.kind("flat", self.arith), self.nslots)
        if not best and self.nslots >= 1 << 20:
            self.min_blocks = 4          # untuned: a register cap (64) rather than the compiler's ~100
        if best:
            self.warps, self.min_blocks = int(best["warps"]), int(best["min_blocks"])
            g = int(best.get("segments", 0))
            self.segments = g if g == 0 or self.brick_h % g == 0 else 0
        self._graph_cache = {}
        self._dtp_dev = None
        self.t = 0.0
        self.nsteps = 0
        self.kernel_launches = 0
        self.halo = None
        self.flat_halo = None
        lam = L.GswLoopState.lam_bits.offset // 8
        self._lam_view = self._state.view(torch.int64)[lam:lam + 1]   # the wave-speed bits

    # ------------------------------------------------------------- forcings
    def set_rain(self, rain):
        """Attach a RainfallForcing (uniform or (nt, nx, ny) gridded)."""
        if rain is None:
            self._rain, self._rain_kind, self._rain_t = None, L.RAIN_NONE, None
            self._rain_lookup, self._rain_ncol = None, 0
            self._graph_cache.clear()
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

    def _set_rain_table(self, t_s, table, lookup_slots):
        """Rain as the reference's flat bundle: a (nt, ncol) table of rates (m/s), the
        frame times, and per slot the column it reads (compressed_solver.py:3273-3282)."""
        self._rain = torch.from_numpy(np.ascontiguousarray(table, np.float32)).to(self.device)
        self._rain_t = torch.from_numpy(np.asarray(t_s, np.float64).copy()).to(self.device)
        self._rain_kind = L.RAIN_LOOKUP
        self._rain_lookup = lookup_slots.to(torch.int32).contiguous()
        self._rain_ncol = int(table.shape[1])
        self._rain_rmax = float(np.max(table)) if table.size else 0.0
        self._graph_cache.clear()

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
            if self.flat_halo is not None:
                gi, gj = self.ij_active[g, 0], self.ij_active[g, 1]
                h, w = self.ngh, self.halo
                seam = ((w.has_neighbor("x-") & (gi < h)) | (w.has_neighbor("x+") & (gi >= self.nxp - h)) |
                        (w.has_neighbor("y-") & (gj < h)) | (w.has_neighbor("y+") & (gj >= self.nyp - h)))
                if seam.any():
                    raise ValueError("add_inflow: a ghost cell lies in a seam ghost strip, which the neighbouring "
                                     "rank owns; list the inlet cells of this rank's own block")
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

    # ----------------------------------------------- per-step coastal forcings
    def _slots_of_padded(self, rows, cols):
        """Slots of padded (i, j) cells (-1 where the cell is not stored)."""
        i = torch.as_tensor(np.asarray(rows, np.int64), device=self.device)
        j = torch.as_tensor(np.asarray(cols, np.int64), device=self.device)
        lut = torch.full((self.nxp * self.nyp,), -1, dtype=torch.int64, device=self.device)
        lut[self._lin_of_slot.to(torch.int64)] = self._slot_cells.to(torch.int64)
        return lut[i * self.nyp + j].contiguous()

    def _pack_padded(self, field, dtype):
        f = torch.as_tensor(np.ascontiguousarray(np.asarray(field)), device=self.device).reshape(-1)
        out = torch.zeros(self.nslots, dtype=dtype, device=self.device)
        out[self._slot_cells] = f[self._lin_of_slot].to(dtype)
        return out

    def set_sponge(self, sponge):
        """Open-boundary sponge (compressed_solver.py:3148-3156): {"keep": k, "amb": a} on
        the padded grid; each step h <- keep*h + amb, hu, hv <- keep*hu, keep*hv over the
        band where keep != 1 or amb != 0."""
        self._forcing.pop("sponge", None)
        if sponge is not None:
            keep = np.asarray(sponge["keep"], np.float32)
            amb = np.asarray(sponge["amb"], np.float32)
            if keep.shape != (self.nxp, self.nyp) or amb.shape != keep.shape:
                raise ValueError(f"set_sponge: keep and amb must be padded ({self.nxp}, {self.nyp}) fields")
            ii, jj = np.nonzero((keep != 1.0) | (amb != 0.0))
            slots = self._slots_of_padded(ii, jj)
            ok = (slots >= 0).cpu().numpy()
            self._forcing["sponge"] = dict(slots=slots[torch.from_numpy(ok).to(self.device)].contiguous(),
                                           keep=torch.from_numpy(keep[ii[ok], jj[ok]].copy()).to(self.device),
                                           amb=torch.from_numpy(amb[ii[ok], jj[ok]].copy()).to(self.device))
        self._graph_cache.clear()
        return self

    def set_infil(self, infil):
        """Landcover infiltration (compressed_solver.py:3212, infiltrate_flat): {"tab":
        rate (m/s) per Manning class}; each step h <- max(h - tab[class] dt, 0) with the
        velocity kept."""
        self._forcing.pop("infil", None)
        if infil is not None:
            self._forcing["infil"] = torch.from_numpy(np.asarray(infil["tab"], np.float32).reshape(-1).copy()
                                                      ).to(self.device)
        self._graph_cache.clear()
        return self

    def set_ga_drain(self, b):
        """Green-Ampt infiltration and linear-reservoir drain (compressed_solver.py:3214,
        3284-3292): {cls_pad, Ks_t, psi_t, dth_t, F_pad, Fmax_pad?, inv_tau_pad?, mode}
        with padded per-cell fields and per-class tables; mode "fused", "ga" or "drain"."""
        self._forcing.pop("ga", None)
        if b is not None:
            mode = {"fused": 1, "ga": 2, "drain": 3}[b.get("mode", "fused")]
            t = lambda k: torch.from_numpy(np.asarray(b[k], np.float32).reshape(-1).copy()).to(self.device)
            self._forcing["ga"] = dict(
                mode=mode, cls=self._pack_padded(b["cls_pad"], torch.uint8),
                Ks=t("Ks_t"), psi=t("psi_t"), dth=t("dth_t"), F=self._pack_padded(b["F_pad"], torch.float32),
                Fmax=(self._pack_padded(b["Fmax_pad"], torch.float32) if b.get("Fmax_pad") is not None else None),
                inv_tau=(self._pack_padded(b["inv_tau_pad"], torch.float32)
                         if b.get("inv_tau_pad") is not None else None))
            if mode != 2 and self._forcing["ga"]["inv_tau"] is None:
                raise ValueError("set_ga_drain: the drain needs inv_tau_pad")
        self._graph_cache.clear()
        return self

    def set_clamp(self, b):
        """Stage clamp (compressed_solver.py:3216, 3294-3299): {rows, cols, hmax} padded
        cells where h is capped at hmax with the velocity kept."""
        self._forcing.pop("clamp", None)
        if b is not None and len(b["rows"]) > 0:
            self._forcing["clamp"] = dict(slots=self._slots_of_padded(b["rows"], b["cols"]),
                                          hmax=torch.from_numpy(np.asarray(b["hmax"], np.float32).copy()
                                                                ).to(self.device))
        self._graph_cache.clear()
        return self

    def set_drain(self, drain):
        """Karst drain cap (compressed_solver.py:3211, drain_cap): {idx (canonical flat
        ids), h_tgt or h_tgt_arr}; h is capped at the target with the velocity kept."""
        self._forcing.pop("drain", None)
        if drain is not None:
            idx = torch.from_numpy(np.asarray(drain["idx"], np.int64).reshape(-1)).to(self.device)
            ht = (np.asarray(drain["h_tgt_arr"], np.float32) if "h_tgt_arr" in drain
                  else np.full(idx.numel(), np.float32(drain.get("h_tgt", 0.5)), np.float32))
            self._forcing["drain"] = dict(slots=self._slot[idx].contiguous(),
                                          htgt=torch.from_numpy(ht.reshape(-1).copy()).to(self.device))
        self._graph_cache.clear()
        return self

    def _forcing_args(self, q, phase):
        f = self._forcing
        a = L.GswFlatForcingArgs()
        a.abi_version = L.ABI_VERSION
        a.phase = phase
        a.q0, a.q1, a.q2, a.flags = _ptr(q[0]), _ptr(q[1]), _ptr(q[2]), _ptr(self._flags)
        a.nslots, a.h_min, a.state = self.nslots, self.h_min, _ptr(self._state)
        if phase == 0:
            if "infil" in f:
                a.n_cls, a.infil_tab = _ptr(self._ncls), _ptr(f["infil"])
            if "sponge" in f:
                sp = f["sponge"]
                a.sp_slots, a.sp_keep, a.sp_amb, a.sp_n = (_ptr(sp["slots"]), _ptr(sp["keep"]), _ptr(sp["amb"]),
                                                           int(sp["slots"].numel()))
        else:
            if "ga" in f:
                g = f["ga"]
                a.ga_mode, a.ga_cls, a.Ks_t, a.psi_t, a.dth_t = (g["mode"], _ptr(g["cls"]), _ptr(g["Ks"]),
                                                                 _ptr(g["psi"]), _ptr(g["dth"]))
                a.F, a.Fmax, a.inv_tau = _ptr(g["F"]), _ptr(g["Fmax"]), _ptr(g["inv_tau"])
            if "clamp" in f:
                a.cl_slots, a.cl_hmax, a.cl_n = (_ptr(f["clamp"]["slots"]), _ptr(f["clamp"]["hmax"]),
                                                 int(f["clamp"]["slots"].numel()))
            if "drain" in f:
                a.dr_slots, a.dr_htgt, a.dr_n = (_ptr(f["drain"]["slots"]), _ptr(f["drain"]["htgt"]),
                                                 int(f["drain"]["slots"].numel()))
        return a

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

    def _inlet_dry_seeds(self):
        """Each inlet's dry-seed reductions over the ranks (inlet_dry_reductions), once per
        inlet list (the bed does not change), kept with the inlet as `dry` for the apply
        kernel."""
        if all("dry" in f for f in self._inflows):
            return
        zb = [self._b[f["nbr"]].cpu().numpy().astype(np.float32) for f in self._inflows]
        for f, d in zip(self._inflows, inlet_dry_reductions(zb, self.halo, self.device)):
            f["dry"] = torch.tensor(d, dtype=torch.float64, device=self.device)

    def _inflow_args(self, f, q, hsum=None):
        a = L.GswFlatInflowArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = L.F32
        a.q0, a.q1, a.q2, a.bed = _ptr(q[0]), _ptr(q[1]), _ptr(q[2]), _ptr(self._b)
        a.ghost_slot, a.nbr_slot, a.n = _ptr(f["ghost"]), _ptr(f["nbr"]), f["n"]
        a.nx_n, a.ny_n, a.ds = f["nx"], f["ny"], f["ds"]
        a.t_knots, a.q_knots, a.n_knots = _ptr(f["t"]), _ptr(f["q"]), int(f["t"].numel())
        a.state = _ptr(self._state)
        a.hsum = hsum
        a.dry = _ptr(f["dry"]) if "dry" in f else None
        return a

    # ---------------------------------------------------------------- views
    def _canonical(self):
        """The reference's CompressedSWE tables of this mesh (host, bit-exact), built on
        first use: ij_active (N, 2), nbr (N, 4) int16 deltas, is_active (N)."""
        if self._tables_cache is None:
            t = build_tables(self._inside.cpu().numpy(), ring=2)
            assert t["N"] == self.N_stored
            # the cells this solver updates: on a split run its own inside cells, not the
            # neighbours' inside cells stored in its seam ghost rows
            t["is_active"] = ((self._flags[self._slot] & SLOT_ACTIVE) != 0).cpu().numpy().astype(np.uint8)
            self._tables_cache = t
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
        a.warps, a.min_blocks, a.segments = self.warps, self.min_blocks, self.segments
        a.arith = self.arith
        if step:
            a.state = _ptr(self._state)
            a.lam_target = C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset)
            a.rain_kind = self._rain_kind
            a.rain = _ptr(self._rain)
            a.rain_lookup, a.rain_ncol = _ptr(self._rain_lookup), int(self._rain_ncol)
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

    def run(self, t_end=None, *, dt_max=None, max_steps: int = 10 ** 9, window: int = 0, say=None,
            checkpoint_every_s: float = 0.0, ckpt_dir=None, resume: bool = False, **unused):
        """Step from the current time to ``t_end`` (the reference's flat loop,
        compressed_solver.py:2133-2448): dt from the previous step's wave speed, the rain
        film limit folded into dt_max, dt = min(dt, t_end - t). Returns the number of steps.

        Checkpoints (compressed_solver.py:1789-1936): with ``checkpoint_every_s`` and
        ``ckpt_dir`` the state, time and step count are written in the reference's format
        (ckpt_r00.npz + ckpt_meta.json, each replaced atomically) at the first window
        boundary past every interval, and once more at the end; ``resume=True`` first
        restores the checkpoint in ``ckpt_dir`` if there is one. A resumed run continues
        the uninterrupted trajectory bit for bit (checkpoints sit on step boundaries and
        do not clip dt)."""
        if t_end is None:
            raise TypeError("CompressedSolver.run() needs t_end, the end time in seconds")
        if resume and ckpt_dir is not None:
            self.load_checkpoint(ckpt_dir, missing_ok=True)
        every = float(checkpoint_every_s or 0.0)
        if every > 0.0 and ckpt_dir is None:
            raise ValueError("CompressedSolver.run: checkpoint_every_s needs ckpt_dir")
        next_ckpt = self.t + every if every > 0.0 else float("inf")
        steps0 = self.nsteps
        if self._rain is None and self._dense_had_rain:
            warnings.warn("CompressedSolver.run: the dense Config asked for rainfall and none was attached "
                          "here. from_dense does not carry rainfall over; pass the same RainfallForcing "
                          "to set_rain().", stacklevel=2)
        dm = dt_max if dt_max is not None else self.dt_max_user
        split = self.flat_halo is not None
        inlet_sums = None
        if split:
            # one sum collective per step when there are inlets: every rank must list the
            # same inlets (compressed_solver.py:2117-2121; entries may hold no local cells)
            self.halo.check_same(len(self._inflows), "CompressedSolver: discharge inlets")
            if self._inflows:
                inlet_sums = torch.zeros(len(self._inflows), dtype=torch.float64, device=self.device)
                self._inlet_dry_seeds()
        K = int(window) if window else self._window_size()
        if split and not window:
            K = min(K, 32)     # launched eagerly: poll often, so few no-op steps follow the end
        if max_steps and max_steps < K and not window:
            K = int(max_steps)
        K += K % 2
        self._write_state()
        self._lammax_into_state()
        p = self._dt_params(t_end, dm, max_steps)
        # the dt rule is read from device memory, so one captured window serves every
        # t_end / dt_max / max_steps
        if self._dtp_dev is None:
            self._dtp_dev = torch.zeros(C.sizeof(L.GswDtParams), dtype=torch.uint8, device=self.device)
        L.call("gsw_dt_params_upload", C.byref(p), _ptr(self._dtp_dev), _stream())
        start = self._cur
        _host_lib()

        forced = bool(self._forcing)
        per_step = 2 + len(self._inflows) + (self._ring is not None) + 3 * forced
        if split:
            per_step += self.flat_halo.launches_per_exchange + (len(self._inflows) if inlet_sums is not None else 0)
        nb_in = self.n_bricks_inner
        if split:                               # the step in two brick ranges
            per_step += int(nb_in > 0) + int(self.n_bricks > nb_in) - 1

        def one_step(k_parity):
            s = _stream()
            if split:                           # every rank takes the dt of the largest wave speed
                self.halo.allreduce_max_(self._lam_view)
            L.call("gsw_dt_finalize_dev", _ptr(self._dtp_dev), _ptr(self._state), s)
            src, dst = self._q[k_parity], self._q[1 - k_parity]
            sums = [None] * len(self._inflows)
            if inlet_sums is not None:          # an inlet may span ranks: one batched sum of
                base = inlet_sums.data_ptr()    # every inlet's depth over the ranks (:2145-2153)
                sums = [C.c_void_p(base + 8 * k) for k in range(len(self._inflows))]
                for f, p in zip(self._inflows, sums):
                    L.call("gsw_flat_inflow_depth_sum", C.byref(self._inflow_args(f, src)), p, s)
                self.halo.allreduce_sum_(inlet_sums)
            for f, p in zip(self._inflows, sums):   # inlet ghosts at t_n, before the step
                L.call("gsw_flat_inflow_apply", C.byref(self._inflow_args(f, src, p)), s)
            a = self._args(src, dst)
            if forced:                          # the wave speed is taken after the forcings
                a.lam_target = None
            if split:
                # seam ghosts from the neighbours (the reference posts them before its
                # interior step, compressed_solver.py:2185-2190, 2209-2222): the bricks
                # that read no seam ghost cell step while the transfer is in flight, the
                # rest after the ghosts are in place
                hnd = self.flat_halo.start(src)
                a.brick_lo, a.brick_hi = 0, nb_in
                if nb_in:
                    L.call("gsw_flat_step", C.byref(a), s)
                self.flat_halo.finish(hnd)
                a.brick_lo, a.brick_hi = nb_in, self.n_bricks
            if not split or self.n_bricks > nb_in:
                L.call("gsw_flat_step", C.byref(a), s)
            if forced:
                L.call("gsw_flat_forcings", C.byref(self._forcing_args(dst, 0)), s)
            if self._ring is not None:          # ring stage at t_n, after the step
                L.call("gsw_flat_ring_stage", C.byref(self._ring_args(dst)), s)
            if forced:
                L.call("gsw_flat_forcings", C.byref(self._forcing_args(dst, 1)), s)
                L.call("gsw_flat_lammax", C.byref(self._args(dst, dst, step=False)),
                       C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset), s)

        def one_window():
            for k in range(K):
                one_step(k % 2)
            return per_step * K

        if start == 1:
            # one step outside the window, so every captured window starts on buffer 0
            one_step(1)
            self.kernel_launches += per_step
        key = (K, self._rain_kind, len(self._inflows), self._ring is not None, self.warps, self.min_blocks,
               self.segments, tuple(sorted(self._forcing)))
        if split:                               # the step sequence holds collectives: eager
            g, per = None, 0
        else:
            g, per = _cached_graph(self._graph_cache, key, one_window, self.device)
        self.kernel_launches += 1
        while True:
            if g is None:
                per = one_window()
            else:
                g.replay()
            self.kernel_launches += per
            st = self._read_state()
            if st.done or _loop_finished(st, p):
                break
            if every > 0.0:
                executed = int(st.steps) + int(st.pending)
                t_now = float(st.t_new) if st.pending else float(st.t)
                if t_now >= next_ckpt:
                    self._write_checkpoint(ckpt_dir, self._q[(start + executed) % 2], t_now, steps0 + executed)
                    while next_ckpt <= t_now:
                        next_ckpt += every
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
        if every > 0.0:
            self._write_checkpoint(ckpt_dir, self._q[self._cur], self.t, self.nsteps)
        return steps

    # ------------------------------------------------------- cache, checkpoints
    def _canonical_of_slot(self):
        c = torch.full((self.nslots,), -1, dtype=torch.int64, device=self.device)
        c[self._slot] = torch.arange(self.N_stored, device=self.device)
        return c

    def _write_checkpoint(self, ckpt_dir, q, t, steps):
        import json
        import os
        os.makedirs(ckpt_dir, exist_ok=True)
        arrays = {f"q{c}": q[c][self._slot].cpu().numpy() for c in range(3)}
        if self._max_h is not None:
            arrays["max_h"] = self._max_h[self._slot].cpu().numpy()
        if "ga" in self._forcing:                  # Green-Ampt's cumulative infiltration is state
            arrays["F"] = self._forcing["ga"]["F"][self._slot].cpu().numpy()
        rank, nranks = self._rank_and_size()
        tmp = os.path.join(ckpt_dir, f"ckpt_r{rank:02d}_tmp")
        np.savez(tmp, t=np.float64(t), steps=np.int64(steps), **arrays)
        os.replace(tmp + ".npz", os.path.join(ckpt_dir, f"ckpt_r{rank:02d}.npz"))
        # a split run: every rank's state file is in place before rank 0 publishes the
        # meta (compressed_solver.py:1861-1866), so the pair on disk is never torn
        if nranks > 1:
            self._barrier()
        if rank == 0:
            meta = dict(t=float(t), steps=int(steps), fidx=0, next_frame=0.0, nranks=nranks)
            mt = os.path.join(ckpt_dir, "ckpt_meta.json.tmp")
            with open(mt, "w") as f:
                json.dump(meta, f)
            os.replace(mt, os.path.join(ckpt_dir, "ckpt_meta.json"))
        if nranks > 1:
            self._barrier()

    def _placement(self):
        """This block's place in the global grid, from every rank's block extents (one
        all-gather): ({i0, j0, nx_loc, ny_loc}, (nx_glob, ny_glob))."""
        import torch.distributed as dist
        h = self.halo
        dev = h.device if h.device_direct else torch.device("cpu")
        mine = torch.tensor([h.coords[0], h.coords[1], self.nx, self.ny], dtype=torch.int64, device=dev)
        every = [torch.zeros_like(mine) for _ in range(h.size)]
        dist.all_gather(every, mine, group=h.group)
        blocks = [tuple(int(v) for v in t.cpu()) for t in every]
        cx, cy = h.coords
        i0 = sum(b[2] for b in blocks if b[1] == cy and b[0] < cx)
        j0 = sum(b[3] for b in blocks if b[0] == cx and b[1] < cy)
        nxg = sum(b[2] for b in blocks if b[1] == cy)
        nyg = sum(b[3] for b in blocks if b[0] == cx)
        return dict(i0=int(i0), j0=int(j0), nx_loc=int(self.nx), ny_loc=int(self.ny)), (int(nxg), int(nyg))

    def _rank_and_size(self):
        if self.flat_halo is None:
            return 0, 1
        return int(self.halo.rank), int(self.halo.size)

    def _barrier(self):
        import torch.distributed as dist
        dist.barrier(group=self.halo.group)

    def load_checkpoint(self, ckpt_dir, missing_ok: bool = False):
        """Restore state, time and step count from a checkpoint in the reference's format
        (ckpt_meta.json + ckpt_r##.npz, one state file per rank of a split run; resumed with
        the same rank count, compressed_solver.py:1881-1895). Returns False when there is
        none and `missing_ok`."""
        import json
        import os
        rank, nranks = self._rank_and_size()
        mp = os.path.join(ckpt_dir, "ckpt_meta.json")
        if not os.path.exists(mp):
            if missing_ok:
                return False
            raise FileNotFoundError(mp)
        meta = json.load(open(mp))
        if int(meta.get("nranks", 1)) != nranks:
            raise RuntimeError(f"checkpoint nranks={meta['nranks']} != current nranks={nranks}; resume with the "
                               f"same rank count (per-rank states are tied to the partition)")
        z = np.load(os.path.join(ckpt_dir, f"ckpt_r{rank:02d}.npz"))
        if "t" in z.files and (abs(float(z["t"]) - float(meta["t"])) > 1e-9 or int(z["steps"]) != int(meta["steps"])):
            raise RuntimeError("torn checkpoint: the state file and ckpt_meta.json disagree on (t, steps)")
        for c in range(3):
            qc = np.asarray(z[f"q{c}"], np.float32).reshape(-1)
            if qc.size != self.N_stored:
                raise ValueError(f"checkpoint has {qc.size} cells, the mesh {self.N_stored}")
            self._q[self._cur][c][self._slot] = torch.from_numpy(qc).to(self.device)
        if self._max_h is not None:
            if "max_h" in z.files:
                self._max_h[self._slot] = torch.from_numpy(np.asarray(z["max_h"], np.float32)).to(self.device)
            else:
                warnings.warn("load_checkpoint: no max_h in the checkpoint; the max-depth envelope only "
                              "covers the resumed window", RuntimeWarning, stacklevel=2)
        if "ga" in self._forcing:
            if "F" not in z.files:
                raise RuntimeError("resume: Green-Ampt is active but the checkpoint has no F array; resuming "
                                   "would reset cumulative infiltration to zero")
            self._forcing["ga"]["F"][self._slot] = torch.from_numpy(np.asarray(z["F"], np.float32)).to(self.device)
        self.t = float(meta["t"])
        self.nsteps = int(meta["steps"])
        return True

    def save_cache(self, cache_dir, *, x0: float = 0.0, y0: float = 0.0, crs_wkt: str = "",
                   nx_glob: Optional[int] = None, ny_glob: Optional[int] = None):
        """Write the mesh, state, Manning table and the rain / ring bundles in the
        reference's cache format (save_cache, compressed_solver.py:2504-2560), which its
        run_cached and from_cache here both read. Inlets are not part of the format (the
        reference passes them to run_cached).

        A run split over ranks writes one ``r##`` directory per rank (every rank calls
        this), as the reference does under MPI (compressed_solver.py:3342-3356,
        2550-2557): its own cells (`is_active` marks the cells this rank updates), the
        block's placement in the global grid, and each seam face's neighbour, width and
        send / receive cells (canonical ids, row offset, position along the face), in the
        reference's face order."""
        import json
        import os
        split = self.flat_halo is not None
        placement = None
        if split:
            rank, nranks = self._rank_and_size()
            placement, glob = self._placement()
            cache_dir = os.path.join(cache_dir, f"r{rank:02d}")
            if nx_glob is None:
                nx_glob = glob[0]
            if ny_glob is None:
                ny_glob = glob[1]
        os.makedirs(cache_dir, exist_ok=True)
        sv = lambda n, a: np.save(os.path.join(cache_dir, n + ".npy"), np.asarray(a))
        tab = self._canonical()
        N = self.N_stored
        sl = self._slot
        sv("nbr", tab["nbr"]); sv("is_active", tab["is_active"]); sv("ij_active", tab["ij"])
        q = self._q[self._cur]
        for c in range(3):
            sv(f"q{c}", q[c][sl].cpu().numpy().astype(np.float32))
        sv("bed_f", self._b[sl].cpu().numpy().astype(np.float32))
        sv("sig_f", np.zeros(N, np.float32)); sv("inv_sig_f", np.ones(N, np.float32))
        mc = self._ncls[sl].cpu().numpy() if self._ncls is not None else np.zeros(N, np.uint8)
        sv("mcls_f", mc.astype(np.uint8)); sv("m_tab", self._ntab.cpu().numpy().astype(np.float32))
        meta = dict(nxp=self.nxp, nyp=self.nyp, ngh=self.ngh, dx=self.dx, x0=float(x0), y0=float(y0),
                    crs_wkt=str(crs_wkt), nx_glob=int(nx_glob if nx_glob is not None else self.nx),
                    ny_glob=int(ny_glob if ny_glob is not None else self.ny), has_ring=self._ring is not None,
                    has_sponge=False, has_rain=self._rain is not None, no_sigma=True, N=int(N),
                    nranks=int(self._rank_and_size()[1]), mpi=split)
        if split:
            meta["placement"] = placement
            meta["halo_faces"] = []
            canon = self._canonical_of_slot()
            for fi, side in enumerate(s for s in HALO_FACE_ORDER if self.halo.has_neighbor(s)):
                f = self.flat_halo.faces[side]
                P = int(f["P"])
                for k in ("s", "r"):
                    pos = f[k + "pos"]
                    sv(f"halo_f{fi}_{k}fi", canon[f[k + "slot"]].cpu().numpy().astype(np.int32))
                    sv(f"halo_f{fi}_{k}off", (pos // P).cpu().numpy().astype(np.int32))
                    sv(f"halo_f{fi}_{k}perp", (pos % P).cpu().numpy().astype(np.int32))
                meta["halo_faces"].append(dict(nbr=int(self.halo._neighbor(side)), P=P))
        if self._rain is not None:
            table = self._rain.cpu().numpy().astype(np.float32)
            if self._rain_kind == L.RAIN_UNIFORM:
                table, lookup = table.reshape(-1, 1), np.zeros(N, np.int32)
            elif self._rain_kind == L.RAIN_GRIDDED:
                ij = tab["ij"].astype(np.int64)
                ii, jj = ij[:, 0] - self.ngh, ij[:, 1] - self.ngh
                inner = (ii >= 0) & (ii < self.nx) & (jj >= 0) & (jj < self.ny)
                lookup = np.where(inner, ii * self.ny + jj, 0).astype(np.int32)
                table = table.reshape(table.shape[0], -1)
            else:
                lookup = self._rain_lookup[sl].cpu().numpy().astype(np.int32)
            sv("rain_native_rate_dev", table); sv("rain_lookup_flat", lookup)
            sv("rain_t_s", self._rain_t.cpu().numpy())
        if self._ring is not None:
            r = self._ring
            canon = self._canonical_of_slot()
            rs = r["slots"]
            rflat = torch.where(rs >= 0, canon[rs.clamp_min(0)], torch.full_like(rs, -1))
            sv("ring_rflat", rflat.cpu().numpy().astype(np.int32)); sv("ring_rbed", r["bed"].cpu().numpy())
            sv("ring_rwg", r["wg"].cpu().numpy().reshape(-1)); sv("ring_t_common", r["t"].cpu().numpy())
            sv("ring_stage_all", r["stage"].cpu().numpy())
            meta["ring_NG"], meta["ring_n"] = int(r["NG"]), int(r["n"])
        with open(os.path.join(cache_dir, "meta.json"), "w") as f:
            json.dump(meta, f)
