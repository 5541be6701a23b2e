"""Gradients of a gauge-misfit loss through many compressed-mesh steps.

The reference has no adjoint; this module differentiates the flat tier's step
(CompressedSolver's loop: inlet ghosts, fused SRM-HLLC/rain/Euler/wet-dry/Manning step)
with respect to the Manning class table, a scale on the rain rate and the knots of an
inlet hydrograph, for calibration against gauge records.

* Forward (recording) pass: the flat loop on the device with the CFL rule, logging
  every step's dt and the gauge depths of the loss window, and storing the states the
  checkpoint schedule asks for first.
* Reverse sweep: binomial checkpointing (the recursive treeverse schedule of Griewank,
  1992, as in Griewank and Walther's "revolve": with s snapshots and at most t forward
  recomputations of any step, up to C(s+t, s) steps are reversed). States are
  recomputed from snapshots with the recorded dt schedule replayed (GswDtParams mode
  2), and each step is reversed by gsw_adj_flat_step / gsw_adj_flat_inflow /
  gsw_gauge_adjoint with dt and every branch of the forward step held fixed.
* `CalibrationLoss` wraps both in a torch.autograd.Function: loss = L(n_tab, rain_scale,
  knots); backward() runs the reverse sweep.

The loss is L = sum over the last `window` states and the gauges of
(depth - target)^2, state n being the state after n steps (n = N - window + 1 .. N).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from .compressed import CompressedSolver
from .solver import _ptr, _stream


def binomial_beta(s: int, t: int) -> int:
    """Steps reversible with s snapshots and at most t forward recomputations of a step."""
    return math.comb(s + t, s)


def treeverse_split(length: int, s: int) -> int:
    """Offset of the next snapshot when reversing `length` steps with `s` free snapshots.
    With t the smallest count with beta(s, t) >= length, any offset m with a right part
    length - m <= beta(s-1, t) and a left part m <= beta(s, t-1) keeps t recomputations;
    within that range the right part is set to beta(s-1, t-1), which gives the minimal
    total number of forward steps, t*length - beta(s+1, t-1) (to within one step)."""
    if length <= 1 or s <= 0:
        return 0
    t = 0
    while binomial_beta(s, t) < length:
        t += 1
    lo = max(1, length - binomial_beta(s - 1, t))
    hi = min(binomial_beta(s, t - 1), length - 1) if t > 0 else length - 1
    m = length - binomial_beta(s - 1, t - 1) if t > 0 else lo
    return min(max(m, lo), max(hi, lo))


def snapshot_chain(n_steps: int, s: int) -> list:
    """The snapshots treeverse(0, n_steps, s) stores before its first reverse step (the
    rightmost path); a recording pass stores them on the way."""
    chain, n0 = [], 0
    while n_steps - n0 > 1 and s > 0:
        m = n0 + treeverse_split(n_steps - n0, s)
        chain.append(m)
        n0, s = m, s - 1
    return chain


class Treeverse:
    """The reverse sweep of `n_steps` steps with `snapshots` snapshot slots, driven by
    callbacks: store(n) keeps the current state as snapshot n, restore(n) makes snapshot
    n the current state, advance(n0, n1) steps the current state from n0 to n1, free(n)
    drops a snapshot, reverse(n) reverses step n from the current state (the state n).
    Snapshot 0 (the initial state) is always available and not counted; `stored` lists
    snapshots a recording pass already holds."""

    def __init__(self, n_steps, snapshots, store, restore, advance, free, reverse, stored=()):
        self.n, self.s = int(n_steps), int(snapshots)
        self.store, self.restore, self.advance = store, restore, advance
        self.free, self.reverse = free, reverse
        self.stored = set(stored) | {0}
        self.forward_steps = 0
        self.max_live = len(self.stored) - 1
        self.order = []

    def run(self):
        self._tv(0, self.n, self.s)

    def _adv(self, n0, n1):
        if n1 > n0:
            self.advance(n0, n1)
            self.forward_steps += n1 - n0

    def _rev(self, n):
        self.reverse(n)
        self.order.append(n)

    def _tv(self, n0, n1, s):
        if n1 - n0 == 1:
            self.restore(n0)
            self._rev(n0)
            return
        if s <= 0:
            for k in range(n1 - 1, n0 - 1, -1):
                self.restore(n0)
                self._adv(n0, k)
                self._rev(k)
            return
        m = n0 + treeverse_split(n1 - n0, s)
        if m not in self.stored:
            self.restore(n0)
            self._adv(n0, m)
            self.store(m)
            self.stored.add(m)
            self.max_live = max(self.max_live, len(self.stored) - 1)
        self._tv(m, n1, s - 1)
        self.free(m)
        self.stored.discard(m)
        self._tv(n0, m, s)


@dataclass
class Inlet:
    """A discharge inlet: ghost/active pairs (canonical ids), inward normal, cell width
    and the knot times of its hydrograph (the knot values are parameters)."""
    ghost: np.ndarray
    nbr: np.ndarray
    normal: tuple
    ds: float
    t_knots: np.ndarray


def interp_weights(t, xp):
    """W (len(t), len(xp)) with np.interp(t, xp, fp) == W @ fp for every fp."""
    t = np.asarray(t, np.float64)
    xp = np.asarray(xp, np.float64)
    W = np.zeros((t.size, xp.size))
    for i, x in enumerate(t):
        if xp.size == 1 or x <= xp[0]:
            W[i, 0] = 1.0
        elif x >= xp[-1]:
            W[i, -1] = 1.0
        else:
            j = int(np.searchsorted(xp, x, "right") - 1)
            w = (x - xp[j]) / (xp[j + 1] - xp[j])
            W[i, j] += 1.0 - w
            W[i, j + 1] += w
    return W


class FlatAdjoint:
    """Loss and gradients of a gauge misfit over `n_steps` steps of a compressed mesh.

    ``cs`` supplies the mesh, bed, Manning classes and initial state (it is not
    advanced). ``dtype`` float32 is the production path; float64 runs the same kernels
    in double for derivative checks. ``rain_times``/``rain_base`` (m/s) is a uniform
    hyetograph scaled by the rain-scale parameter; ``inlet`` is optional."""

    def __init__(self, cs: CompressedSolver, *, gauges: Sequence[int], n_steps: int, window: int,
                 snapshots: int = 55, dtype: str = "float32", rain_times=None, rain_base=None,
                 inlet: Optional[Inlet] = None):
        if getattr(cs, "flat_halo", None) is not None:
            raise NotImplementedError("FlatAdjoint: the adjoint of a run split over ranks is not supported")
        if window < 1 or window > n_steps:
            raise ValueError("window must be in [1, n_steps]")
        if dtype not in ("float32", "float64"):
            raise ValueError("dtype must be float32 or float64")
        if cs.arith == L.ARITH_FAST:
            raise ValueError("FlatAdjoint: the adjoint differentiates the exact step; build the solver "
                             "with arith='exact' (or 'portable')")
        self.cs = cs
        self.dev = cs.device
        self.adj_min_blocks = 8          # register cap of the binary32 reverse kernels: 0, 6 (80) or 8 (64 regs)
        self.code = L.F32 if dtype == "float32" else L.F64
        self.td = torch.float32 if dtype == "float32" else torch.float64
        self.N, self.K, self.S = int(n_steps), int(window), int(snapshots)
        self.first = self.N - self.K + 1
        td, dev = self.td, self.dev
        self.q_init = [cs._q[cs._cur][c].to(td).clone() for c in range(3)]
        self.bed = cs._b.to(td).contiguous()
        self.nslots = cs.nslots
        self.gauge_ids = np.asarray(gauges, np.int64)
        self.G = int(self.gauge_ids.size)
        if self.G and not (cs.is_active[self.gauge_ids] != 0).all():
            raise ValueError("gauges must be active cells")
        self.gauge_slots = cs._slot[torch.from_numpy(self.gauge_ids).to(dev)].to(torch.int64).contiguous()
        self.n_classes = int(cs._ntab.numel())
        if rain_times is None:
            rain_times, rain_base = np.array([0.0]), np.array([0.0])
        self.rain_t = np.asarray(rain_times, np.float64)
        self.rain_base = np.asarray(rain_base, np.float64)
        self._rain_t_dev = torch.from_numpy(self.rain_t.copy()).to(dev)
        self.inlet = inlet
        if inlet is not None:
            self._in_ghost = cs._slot[torch.from_numpy(np.asarray(inlet.ghost, np.int64)).to(dev)].to(torch.int64)
            self._in_nbr = cs._slot[torch.from_numpy(np.asarray(inlet.nbr, np.int64)).to(dev)].to(torch.int64)
            self._in_t = torch.from_numpy(np.asarray(inlet.t_knots, np.float64).copy()).to(dev)
        z = lambda: torch.zeros(self.nslots, dtype=td, device=dev)
        self._buf = [[z() for _ in range(3)] for _ in range(2)]
        self._lam = [[z() for _ in range(3)] for _ in range(2)]
        self._rbar = [z() for _ in range(3)]
        self._snaps = {}
        self._state = torch.zeros(128, dtype=torch.uint8, device=dev)
        self._state_host = torch.zeros(128, dtype=torch.uint8).pin_memory()
        self.dt_tab = torch.zeros(self.N + 1, dtype=torch.float64, device=dev)
        self.series = torch.zeros((self.K, max(self.G, 1)), dtype=torch.float64, device=dev)
        self.kernel_launches = 0
        self._params = None
        self._schedule = False        # a recorded dt schedule exists
        self._ready = False           # the last forward pass left its snapshots and final state

    # ----------------------------------------------------------------- parameters
    def set_params(self, n_tab, rain_scale, knots=None):
        td, dev = self.td, self.dev
        n_tab = np.asarray(n_tab, np.float64).reshape(-1)
        if n_tab.size != self.n_classes:
            raise ValueError(f"n_tab must have {self.n_classes} classes")
        self._ntab = torch.from_numpy(n_tab.copy()).to(td).to(dev).contiguous()
        self.rain_scale = float(rain_scale)
        rates = (self.rain_scale * self.rain_base).astype(np.float32 if td == torch.float32 else np.float64)
        self._rain = torch.from_numpy(np.ascontiguousarray(rates)).to(dev)
        self._rain_max = float(rates.max()) if rates.size else 0.0
        if self.inlet is not None:
            k = np.asarray(knots, np.float64).reshape(-1)
            if k.size != len(self.inlet.t_knots):
                raise ValueError("knots must match the inlet's knot times")
            self._knots = torch.from_numpy(k.copy()).to(dev)
        self._params = True

    # ------------------------------------------------------------------- plumbing
    def _flat_args(self, q, out=None):
        cs = self.cs
        a = L.GswFlatArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = self.code
        a.brick_h, a.n_bricks = cs.brick_h, cs.n_bricks
        a.brick_ij, a.brick_nbr, a.flags = _ptr(cs._bij), _ptr(cs._bnbr), _ptr(cs._flags)
        a.q0, a.q1, a.q2 = _ptr(q[0]), _ptr(q[1]), _ptr(q[2])
        if out is not None:
            a.qn0, a.qn1, a.qn2 = _ptr(out[0]), _ptr(out[1]), _ptr(out[2])
        a.bed = _ptr(self.bed)
        inv = 1.0 / cs.dx
        if self.code == L.F32:
            inv = float(np.float32(inv))
        a.inv_dx = a.inv_dy = inv
        a.g, a.h_min, a.h_min_cfl = cs.g, cs.h_min, cs.h_min_cfl
        a.linf = int(cs.cfl_linf)
        a.ngh, a.nx, a.ny = cs.ngh, cs.nx, cs.ny
        a.state = _ptr(self._state)
        a.lam_target = C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset)
        a.rain_kind = L.RAIN_UNIFORM
        a.rain = _ptr(self._rain)
        a.n_cls, a.n_tab, a.n_tab_len = _ptr(cs._ncls), _ptr(self._ntab), self.n_classes
        a.vcap, a.quadratic, a.keep_h = cs.vcap, int(cs.quad), int(cs.keep_h)
        a.warps, a.min_blocks = cs.warps, (cs.min_blocks if self.code == L.F32 else 0)
        a.segments = cs.segments
        return a

    def _inflow_args(self, q):
        a = L.GswFlatInflowArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = self.code
        a.q0, a.q1, a.q2, a.bed = _ptr(q[0]), _ptr(q[1]), _ptr(q[2]), _ptr(self.bed)
        a.ghost_slot, a.nbr_slot, a.n = _ptr(self._in_ghost), _ptr(self._in_nbr), int(self._in_ghost.numel())
        a.nx_n, a.ny_n = float(self.inlet.normal[0]), float(self.inlet.normal[1])
        a.ds = float(self.inlet.ds)
        a.t_knots, a.q_knots, a.n_knots = _ptr(self._in_t), _ptr(self._knots), int(self._in_t.numel())
        a.state = _ptr(self._state)
        return a

    def _dt_params(self, mode):
        cs = self.cs
        p = L.GswDtParams()
        p.abi_version = L.ABI_VERSION
        p.mode = mode
        p.cfl_dmin = cs.cfl * cs.dx
        p.lam_floor = (cs.g * cs.h_min) ** 0.5
        p.t_end = 1.0e300
        p.eps_end = 1.0e-9
        p.max_steps = self.N
        p.clip_flat = 1
        dm = 0.0
        if self._rain_max > 0.0:                 # the flat loop's rain film limit as dt_max
            dm = (cs.cfl * cs.dx) ** (2.0 / 3.0) / (cs.g * self._rain_max) ** (1.0 / 3.0)
        p.dt_max = dm
        p.rain_t, p.n_rain = _ptr(self._rain_t_dev), int(self._rain_t_dev.numel())
        if mode == 0:
            p.dt_log = _ptr(self.dt_tab)
        else:
            p.dt_table = _ptr(self.dt_tab)
        return p

    def _set_state(self, t, steps):
        """Loop state (t, steps), written synchronously (start of a forward pass)."""
        st = L.GswLoopState()
        st.t = float(t)
        st.steps = int(steps)
        self._state_host.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))),
                                                dtype=torch.uint8))
        self._state.copy_(self._state_host)
        torch.cuda.current_stream().synchronize()

    def _build_state_table(self):
        """Pinned (N + 1, 128) rows: the loop state at the start of step n (t_n, n). Each
        row is its own host memory, so queued copies never see a row rewritten."""
        raw = bytearray()
        for n in range(self.N + 1):
            st = L.GswLoopState()
            st.t = float(self._t_tab[n])
            st.steps = n
            raw += bytes(st) + bytes(128 - C.sizeof(st))
        self._state_tab = torch.frombuffer(raw, dtype=torch.uint8).reshape(self.N + 1, 128).pin_memory()

    def _set_state_n(self, n):
        self._state.copy_(self._state_tab[n], non_blocking=True)

    def _read_state(self):
        torch.cuda.current_stream().synchronize()
        return L.GswLoopState.from_buffer_copy(self._state.cpu().numpy().tobytes()[:C.sizeof(L.GswLoopState)])

    def _gauge_args(self, q0, offset, lam0=None, target=None):
        a = L.GswGaugeArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = self.code
        a.q0, a.slots, a.n, a.offset = _ptr(q0), _ptr(self.gauge_slots), self.G, int(offset)
        a.first, a.count = self.first, self.K
        a.series = _ptr(self.series)
        a.target = _ptr(target)
        a.weight = 1.0
        a.lam0 = _ptr(lam0)
        a.state = _ptr(self._state)
        return a

    def _one_step(self, src, dst, p, record):
        s = _stream()
        L.call("gsw_dt_finalize", C.byref(p), _ptr(self._state), s)
        if self.inlet is not None:
            L.call("gsw_flat_inflow_apply", C.byref(self._inflow_args(src)), s)
        L.call("gsw_flat_step", C.byref(self._flat_args(src, dst)), s)
        n = 2 + (self.inlet is not None)
        if record and self.G:
            L.call("gsw_gauge_record", C.byref(self._gauge_args(dst[0], 1)), s)
            n += 1
        self.kernel_launches += n

    # ----------------------------------------------------------------- forward
    def forward(self, *, replay=False, snapshots=True):
        """Run N steps from the initial state: the recording pass (CFL rule, dt logged),
        or with `replay` the recorded dt schedule. Returns the gauge series (window,
        gauges) as float64."""
        if self._params is None:
            raise RuntimeError("set_params() first")
        if replay and not self._schedule:
            raise RuntimeError("replay needs a recorded dt schedule (run forward() first)")
        for c in range(3):
            self._buf[0][c].copy_(self.q_init[c])
        self._snaps.clear()
        chain = set(snapshot_chain(self.N, self.S)) if snapshots else set()
        self.series.zero_()
        self._set_state(self.cs.t, 0)
        if not replay:
            self.dt_tab.zero_()
            L.call("gsw_flat_lammax", C.byref(self._flat_args(self._buf[0])),
                   C.c_void_p(self._state.data_ptr() + L.GswLoopState.lam_bits.offset), _stream())
        p = self._dt_params(2 if replay else 0)
        cur = 0
        for n in range(self.N):
            self._one_step(self._buf[cur], self._buf[1 - cur], p, True)
            cur = 1 - cur
            if (n + 1) in chain:
                self._snaps[n + 1] = [x.clone() for x in self._buf[cur]]
        L.call("gsw_loop_commit", _ptr(self._state), _stream())
        st = self._read_state()
        if st.error == L.ERR_NONFINITE:
            raise FloatingPointError("non-finite wave speed in the forward pass")
        if int(st.steps) != self.N:
            raise RuntimeError(f"forward pass took {st.steps} steps, expected {self.N}")
        self._final = cur
        if not replay:
            dt = self.dt_tab.cpu().numpy()[: self.N]
            t = np.empty(self.N + 1)
            t[0] = self.cs.t
            for k in range(self.N):              # the device's own accumulation order
                t[k + 1] = t[k] + dt[k]
            self._t_tab = t
            self._build_state_table()
            self._schedule = True
        self._ready = bool(snapshots)
        self.t_end = float(st.t)
        return self.series[:, : self.G].clone()

    def state(self, c=0):
        """Field c of the final state of the last forward pass (slot-indexed)."""
        return self._buf[self._final][c]

    def loss(self, target):
        d = self.series[:, : self.G] - torch.as_tensor(target, dtype=torch.float64, device=self.dev)
        return float((d * d).sum())

    # ----------------------------------------------------------------- reverse
    def gradients(self, target, *, timing=False):
        """Reverse sweep after forward(): (dL/dn_tab (C,), dL/drain_scale, dL/dknots or None).
        With `timing`, CUDA events bracket every reverse step and every recomputation;
        their totals (ms) land in self.timing."""
        if not (self._schedule and self._ready):
            raise RuntimeError("gradients() needs a forward() pass that kept its snapshots")
        dev = self.dev
        tgt = torch.as_tensor(target, dtype=torch.float64, device=dev).contiguous()
        self._tgt = tgt
        self.n_bar = torch.zeros(self.n_classes, dtype=torch.float64, device=dev)
        self.rate_bar = torch.zeros(self.N + 1, dtype=torch.float64, device=dev)
        self.q_bar = torch.zeros(self.N + 1, dtype=torch.float64, device=dev)
        for lam in self._lam:
            for x in lam:
                x.zero_()
        for x in self._rbar:
            x.zero_()
        p2 = self._dt_params(2)
        self._set_state_n(self.N)                # the loss term of the final state seeds lam
        if self.G:
            L.call("gsw_gauge_adjoint", C.byref(self._gauge_args(self._buf[self._final][0], 0,
                                                                 lam0=self._lam[1][0], target=tgt)), _stream())
        work = self._buf
        self._cur = 0

        def restore(n):
            src = self.q_init if n == 0 else self._snaps[n]
            for c in range(3):
                work[0][c].copy_(src[c])
            self._cur = 0

        def store(n):
            self._snaps[n] = [x.clone() for x in work[self._cur]]

        def free(n):
            self._snaps.pop(n, None)

        ev_rev, ev_adv = [], []

        def events():
            e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            e[0].record()
            return e

        def advance(n0, n1):
            e = events() if timing else None
            self._set_state_n(n0)
            for _ in range(n0, n1):
                self._one_step(work[self._cur], work[1 - self._cur], p2, False)
                self._cur = 1 - self._cur
            if timing:
                e[1].record()
                ev_adv.append(e)

        def reverse(n):
            e = events() if timing else None
            self._reverse_step(n, work[self._cur], p2)
            if timing:
                e[1].record()
                ev_rev.append(e)

        tv = Treeverse(self.N, self.S, store, restore, advance, free, reverse, stored=self._snaps.keys())
        tv.run()
        self.recompute_steps = tv.forward_steps
        self.max_snapshots = tv.max_live
        torch.cuda.current_stream().synchronize()
        if timing:
            self.timing = dict(reverse_ms=sum(a.elapsed_time(b) for a, b in ev_rev), reverse_steps=len(ev_rev),
                               recompute_ms=sum(a.elapsed_time(b) for a, b in ev_adv),
                               recompute_steps=tv.forward_steps)
        self._ready = False                      # snapshots used up, final state overwritten
        g_n = self.n_bar.clone()
        idx = np.clip(np.searchsorted(self.rain_t, self._t_tab[: self.N], "right") - 1, 0, len(self.rain_t) - 1)
        rb = self.rate_bar.cpu().numpy()[: self.N]
        g_s = float(np.sum(rb * self.rain_base[idx]))
        g_k = None
        if self.inlet is not None:
            qb = self.q_bar.cpu().numpy()[: self.N]
            g_k = torch.from_numpy(interp_weights(self._t_tab[: self.N], np.asarray(self.inlet.t_knots)).T @ qb)
        return g_n, g_s, g_k

    def _reverse_step(self, n, q, p2):
        """lam_n from lam_{n+1} for state q = q_n (its inlet ghosts are rewritten here)."""
        s = _stream()
        self._set_state_n(n)
        L.call("gsw_dt_finalize", C.byref(p2), _ptr(self._state), s)
        if self.inlet is not None:
            L.call("gsw_flat_inflow_apply", C.byref(self._inflow_args(q)), s)
        a = L.GswFlatAdjArgs()
        a.abi_version = L.ABI_VERSION
        a.min_blocks = self.adj_min_blocks if self.code == L.F32 else 0
        a.f = self._flat_args(q)
        lin, lout = self._lam[1], self._lam[0]
        a.lam_in0, a.lam_in1, a.lam_in2 = _ptr(lin[0]), _ptr(lin[1]), _ptr(lin[2])
        a.lam_out0, a.lam_out1, a.lam_out2 = _ptr(lout[0]), _ptr(lout[1]), _ptr(lout[2])
        a.rbar0, a.rbar1, a.rbar2 = _ptr(self._rbar[0]), _ptr(self._rbar[1]), _ptr(self._rbar[2])
        a.n_bar, a.rate_bar = _ptr(self.n_bar), _ptr(self.rate_bar)
        L.call("gsw_adj_flat_step", C.byref(a), s)
        k = 3
        if self.inlet is not None:
            L.call("gsw_adj_flat_inflow", C.byref(self._inflow_args(q)), _ptr(lout[0]), _ptr(lout[1]),
                   _ptr(lout[2]), _ptr(self.q_bar), s)
            k += 2
        if self.G:
            L.call("gsw_gauge_adjoint", C.byref(self._gauge_args(q[0], 0, lam0=lout[0], target=self._tgt)), s)
            k += 1
        self.kernel_launches += k
        self._lam = [lin, lout]

    def adjoint_state(self, c=0):
        """Field c of the adjoint of the initial state after gradients() (slot-indexed)."""
        return self._lam[1][c]


class CalibrationLoss(torch.autograd.Function):
    """loss = CalibrationLoss.apply(n_tab, rain_scale, knots, problem, target): a
    recording pass of `problem` (a FlatAdjoint) with these parameters; backward runs the
    checkpointed reverse sweep. `knots` may be an empty tensor when there is no inlet."""

    @staticmethod
    def forward(ctx, n_tab, rain_scale, knots, problem, target):
        problem.set_params(n_tab.detach().cpu().double().numpy(), float(rain_scale.detach()),
                           knots.detach().cpu().double().numpy() if problem.inlet is not None else None)
        problem.forward()
        ctx.problem, ctx.target = problem, target
        ctx.shapes = (n_tab.shape, rain_scale.shape, knots.shape, n_tab.dtype, rain_scale.dtype, knots.dtype)
        return torch.tensor(problem.loss(target), dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        gn, gs, gk = ctx.problem.gradients(ctx.target)
        sn, ss, sk, dn, ds, dk = ctx.shapes
        g = float(g)
        out_n = (gn.cpu() * g).reshape(sn).to(dn)
        out_s = torch.tensor(gs * g, dtype=torch.float64).reshape(ss).to(ds)
        out_k = (gk * g).reshape(sk).to(dk) if gk is not None else torch.zeros(sk, dtype=dk)
        return out_n, out_s, out_k, None, None
