"""Batched ensemble: many compressed meshes advanced together by one kernel per step.

Each member is a CompressedSolver (its own mesh, bed, Manning table, rain and end
time). Their brick storages are concatenated into one, with one shared all-zero brick,
and every step is one persistent launch (gsw_ensemble_step) in which warps take bricks
from the whole ensemble; each member keeps its own CFL dt, rain frame and end time,
computed on the device by the block that finishes each step last. Windows of steps are
captured in a CUDA graph. A member's trajectory is bit-identical to running it alone.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np
import torch

from . import _lib as L
from .compressed import BRICK_PITCH, CompressedSolver
from .solver import _ptr, _stream


GswMember = L.GswMember
GswEnsembleArgs = L.GswEnsembleArgs


def _protos():
    return L.lib()


class Ensemble:
    """Advance a list of CompressedSolver members together (all with the same brick_h)."""

    def __init__(self, members: Sequence[CompressedSolver], *, warps: int = 0, grid: int = 0):
        if not members:
            raise ValueError("Ensemble: no members")
        if any(getattr(m, "flat_halo", None) is not None for m in members):
            raise ValueError("Ensemble: a member split over ranks cannot join an ensemble; spread whole "
                             "members over the ranks instead (partition.members_of)")
        bh = {m.brick_h for m in members}
        if len(bh) != 1:
            raise ValueError(f"Ensemble: members must share brick_h (got {sorted(bh)})")
        ar = {m.arith for m in members}
        if len(ar) != 1:
            raise ValueError("Ensemble: members must share their arithmetic ('exact', 'portable' or 'fast')")
        self.arith = ar.pop()
        _protos()
        self.members = list(members)
        self.brick_h = bh.pop()
        self.device = members[0].device
        BS = self.brick_h * BRICK_PITCH
        self.BS = BS
        nbs = [m.n_bricks for m in members]
        self.brick_off = np.concatenate([[0], np.cumsum(nbs)]).astype(np.int64)
        self.n_bricks = int(self.brick_off[-1])
        NB = self.n_bricks
        dev = self.device
        bij, bnbr, bmem = [], [], []
        for k, m in enumerate(members):
            off = int(self.brick_off[k])
            nb = m.n_bricks
            bij.append(m._bij)
            loc = m._bnbr.to(torch.int64)
            bnbr.append(torch.where(loc >= nb, torch.full_like(loc, NB), loc + off).to(torch.int32))
            bmem.append(torch.full((nb,), k, dtype=torch.int32, device=dev))
        self._bij = torch.cat(bij).contiguous()
        self._bnbr = torch.cat(bnbr).contiguous()
        self._bmem = torch.cat(bmem).contiguous()
        self.nslots = (NB + 1) * BS

        def cat(get, dtype):
            parts = [get(m)[: m.n_bricks * BS].to(dtype) for m in members]
            parts.append(torch.zeros(BS, dtype=dtype, device=dev))
            return torch.cat(parts).contiguous()

        self._q = [[cat(lambda m, c=c: m._q[m._cur][c], torch.float32) for c in range(3)],
                   [torch.zeros(self.nslots, dtype=torch.float32, device=dev) for _ in range(3)]]
        self._b = cat(lambda m: m._b, torch.float32)
        self._flags = cat(lambda m: m._flags, torch.uint8)
        self._ncls = cat(lambda m: (m._ncls if m._ncls is not None else
                                    torch.zeros_like(m._flags)), torch.uint8)
        self._max_h = torch.zeros(self.nslots, dtype=torch.float32, device=dev)
        self._tabs = [m._ntab.to(torch.float32).contiguous() for m in members]
        M = len(members)
        self._states = torch.zeros(M * C.sizeof(L.GswLoopState), dtype=torch.uint8, device=dev)
        self._scratch = torch.zeros(4, dtype=torch.int32, device=dev)
        self._all_done = torch.zeros(1, dtype=torch.int32, device=dev)
        # fixed device buffers: captured graphs hold their addresses across runs
        self._members_dev = torch.zeros(M * C.sizeof(GswMember), dtype=torch.uint8, device=dev)
        # running-member brick list, rebuilt on the device when a member finishes
        self._brick_off_dev = torch.from_numpy(self.brick_off.copy()).to(dev)
        self._run = torch.zeros(2 * M + 2, dtype=torch.int64, device=dev)
        self._parity = np.zeros(M, np.int64)       # buffer of each member's current state
        self.warps, self.grid, self.min_blocks, self.segments = int(warps), int(grid), 0, 0
        # every member in the production configuration: the step compiles it in
        self.lean = all(m.quad and m.keep_h and not m.cfl_linf for m in members)
        self.kernel_launches = 0
        self._graph_cache = {}

    # ------------------------------------------------------------------ I/O
    def member_slots(self, k):
        """Global slots of member k's canonical cells."""
        m = self.members[k]
        return m._slot + int(self.brick_off[k]) * self.BS

    def depth(self, k):
        """Depth (nx, ny) of member k, zero outside its active set."""
        m = self.members[k]
        q = self._q[int(self._parity[k])][0]
        off = int(self.brick_off[k]) * self.BS
        out = torch.zeros(m.nxp * m.nyp, dtype=torch.float32, device=self.device)
        act = (m._flags[m._slot_cells] & 2) != 0
        out[m._lin_of_slot[act]] = q[m._slot_cells[act] + off]
        g = m.ngh
        return out.reshape(m.nxp, m.nyp)[g:-g, g:-g].cpu().numpy()

    def flat(self, k, c=0):
        """Field c of member k in the reference's canonical flat order."""
        return self._q[int(self._parity[k])][c][self.member_slots(k)]

    @property
    def active_cells(self):
        return [m.N_active for m in self.members]

    # ---------------------------------------------------------------- running
    def _args(self, src, dst):
        a = GswEnsembleArgs()
        a.abi_version = L.ABI_VERSION
        a.brick_h, a.n_bricks, a.n_members = self.brick_h, self.n_bricks, len(self.members)
        a.warps, a.grid, a.min_blocks, a.segments = self.warps, self.grid, self.min_blocks, self.segments
        a.arith = self.arith
        a.brick_ij, a.brick_nbr, a.brick_member = _ptr(self._bij), _ptr(self._bnbr), _ptr(self._bmem)
        a.flags, a.n_cls = _ptr(self._flags), _ptr(self._ncls)
        a.q0, a.q1, a.q2 = _ptr(src[0]), _ptr(src[1]), _ptr(src[2])
        a.qn0, a.qn1, a.qn2 = _ptr(dst[0]), _ptr(dst[1]), _ptr(dst[2])
        a.bed, a.max_h = _ptr(self._b), _ptr(self._max_h)
        a.members, a.states = _ptr(self._members_dev), _ptr(self._states)
        a.scratch, a.all_done = _ptr(self._scratch), _ptr(self._all_done)
        a.member_brick_off, a.run = _ptr(self._brick_off_dev), _ptr(self._run)
        a.lean = int(self.lean)
        return a

    def _build_members(self, t_end, max_steps, dt_max):
        M = len(self.members)
        arr = (GswMember * M)()
        t_ends = list(t_end) if np.ndim(t_end) else [float(t_end)] * M
        for k, m in enumerate(self.members):
            mb = arr[k]
            mb.dt = m._dt_params(t_ends[k], dt_max, max_steps)
            mb.inv_dx = float(np.float32(1.0 / m.dx))
            mb.g, mb.h_min, mb.h_min_cfl, mb.vcap = m.g, m.h_min, m.h_min_cfl, m.vcap
            mb.linf, mb.quadratic, mb.keep_h = int(m.cfl_linf), int(m.quad), int(m.keep_h)
            mb.g_recip = L.lib().gsw_div_const_recip(float(np.float32(m.g)))   # the flat step's h / g
            if m._rain_kind not in (L.RAIN_NONE, L.RAIN_UNIFORM):
                raise NotImplementedError("Ensemble members take uniform rain (one rate per frame)")
            mb.rain_kind = m._rain_kind
            mb.rain = _ptr(m._rain)
            mb.n_tab = _ptr(self._tabs[k])
        self._members_dev.copy_(torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8))
        st = (L.GswLoopState * M)()
        for k, m in enumerate(self.members):
            st[k].t = float(m.t)
        self._states.copy_(torch.frombuffer(bytearray(bytes(st)), dtype=torch.uint8))

    def read_states(self):
        M = len(self.members)
        raw = self._states.cpu().numpy().tobytes()
        return (L.GswLoopState * M).from_buffer_copy(raw)

    def _prepare(self, t_end, max_steps, dt_max):
        """Members' parameters and fresh loop states, every member's state in one buffer,
        the initial wave speeds reduced and the first dt evaluated. Returns that buffer."""
        M = len(self.members)
        self._build_members(t_end, max_steps, dt_max)
        p0 = int(np.bincount(self._parity, minlength=2).argmax())
        for k in range(M):                       # bring every member's state into buffer p0
            if self._parity[k] != p0:
                a, b = int(self.brick_off[k]) * self.BS, int(self.brick_off[k + 1]) * self.BS
                for c in range(3):
                    self._q[p0][c][a:b].copy_(self._q[1 - p0][c][a:b])
                self._parity[k] = p0
        s = _stream()
        self._scratch.zero_()
        self._all_done.zero_()
        L.call("gsw_ensemble_lammax", C.byref(self._args(self._q[p0], self._q[p0])), s)
        L.call("gsw_ensemble_finalize", C.byref(self._args(self._q[p0], self._q[p0])), s)
        self.kernel_launches += 2
        return p0

    def time_step(self, t_end, *, warps, grid, min_blocks=0, segments=0, reps=6, max_steps: int = 10 ** 9,
                  dt_max=None):
        """Mean duration (ms) of one ensemble step launch with the given schedule, from the
        current state; the states are restored before every launch and the members' state
        is left as it was."""
        _protos()
        p0 = self._prepare(t_end, max_steps, dt_max)
        snap, snap_run = self._states.clone(), self._run.clone()
        saved = (self.warps, self.grid, self.min_blocks, self.segments)
        self.warps, self.grid, self.min_blocks, self.segments = int(warps), int(grid), int(min_blocks), int(segments)
        args = self._args(self._q[p0], self._q[1 - p0])
        self.warps, self.grid, self.min_blocks, self.segments = saved
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total = 0.0
        for k in range(reps + 1):
            self._states.copy_(snap)
            self._run.copy_(snap_run)
            self._scratch.zero_()
            self._all_done.zero_()
            e0.record()
            L.call("gsw_ensemble_step", C.byref(args), _stream())
            e1.record()
            torch.cuda.synchronize()
            if k:
                total += e0.elapsed_time(e1)
        self.kernel_launches += reps + 1
        self._states.copy_(snap)
        self._run.copy_(snap_run)
        return total / reps

    def run(self, t_end, *, max_steps: int = 10 ** 9, dt_max=None, window: int = 64):
        """Advance every member to its t_end (scalar or one per member). Returns the list
        of steps each member took."""
        _protos()
        p0 = self._prepare(t_end, max_steps, dt_max)
        K = int(window) + int(window) % 2

        def one_window():
            st = _stream()
            for k in range(K):
                src, dst = self._q[(p0 + k) % 2], self._q[(p0 + k + 1) % 2]
                L.call("gsw_ensemble_step", C.byref(self._args(src, dst)), st)
            return K

        key = (K, p0, self.warps, self.grid, self.min_blocks, self.segments, self.lean)
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
        host = torch.zeros(1, dtype=torch.int32).pin_memory()
        while True:
            g.replay()
            self.kernel_launches += per
            host.copy_(self._all_done, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            if int(host[0]):
                break
        sts = self.read_states()
        steps = []
        for k, m in enumerate(self.members):
            n = int(sts[k].steps)
            steps.append(n)
            self._parity[k] = (p0 + n) % 2
            m.t = float(sts[k].t)
            m.nsteps += n
            if sts[k].error == L.ERR_NONFINITE:
                raise FloatingPointError(f"ensemble member {k}: non-finite max wave speed at t={m.t:.3f}s")
            if sts[k].error == L.ERR_INVALID:
                raise RuntimeError(f"ensemble member {k} was stopped at t={m.t:.3f}s: the step ran compiled for "
                                   f"the production configuration (Ensemble.lean), which this member does not have")
        return steps
