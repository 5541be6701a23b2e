"""Halo exchange for a Cartesian split of the dense grid over torch.distributed ranks.

Replaces ``Halo2D`` of the reference (geoswe/mpi_halo.py:278-721), which exchanges the
face strips of ``(*, nxp, nyp)`` arrays over an MPI Cartesian communicator, and its
face-extent check (mpi_halo.py:256-275, 361-387). Here the ranks are the members of a
``torch.distributed`` process group, one process per GPU:

* NCCL group: the faces are packed into contiguous device buffers on the current
  stream and moved by one ``batch_isend_irecv`` per exchange (NVLink / NVSwitch between
  the GPUs of a node); waiting on the works orders the current stream after the
  transfers, so nothing synchronises the host.
* any other backend (gloo): the faces of a CUDA array are staged through host buffers,
  as the reference does when its MPI is not GPU-aware; CPU arrays go as they are.

Layout: ``dims = [Px, Py]`` ranks, rank ``r`` at coordinates ``(r // Py, r % Py)`` (the
row-major order of an MPI Cartesian communicator created with ``reorder=False``); the
default ``dims`` is the most nearly square factorisation with ``Px >= Py``
(``MPI.Compute_dims``). A face has a neighbour when the next rank along its axis
exists, or wraps round on a periodic axis that is split (``P > 1``). A periodic axis
that is not split has no neighbour on either face: its wrap is the ghost fill's
periodic copy on this rank, the exchange the reference's size-1 periodic axis does with
itself.

Only the four face strips move; the ``ngh x ngh`` corner blocks are not exchanged
(mpi_halo.py:480-492): the dimensionally split SRM-HLLC stencil never reads them.
"""
from __future__ import annotations

from typing import Optional

import torch
import torch.distributed as dist

__all__ = ["Halo2D", "FlatHalo", "compute_dims", "check_face_extent", "comm_size", "SIDES"]

SIDES = ("x-", "x+", "y-", "y+")
_OPPOSITE = {"x-": "x+", "x+": "x-", "y-": "y+", "y+": "y-"}
# a message's tag is the face it lands in on the receiving rank
_TAG = {"x-": 0, "x+": 1, "y-": 2, "y+": 3}


def comm_size(comm) -> int:
    """Number of ranks of ``comm`` (a torch.distributed process group), 1 for None."""
    if comm is None:
        return 1
    if not isinstance(comm, dist.ProcessGroup):
        raise TypeError(f"comm must be a torch.distributed ProcessGroup (for example "
                        f"torch.distributed.group.WORLD), got {type(comm).__name__}")
    return dist.get_world_size(comm)


def compute_dims(size: int):
    """The most nearly square ``[Px, Py]`` with ``Px * Py == size`` and ``Px >= Py``
    (what ``MPI.Compute_dims(size, 2)`` returns)."""
    size = int(size)
    if size < 1:
        raise ValueError(f"compute_dims: size must be at least 1, got {size}")
    py = 1
    f = 1
    while f * f <= size:
        if size % f == 0:
            py = f
        f += 1
    return [size // py, py]


def check_face_extent(side, nbr, mine, theirs):
    """Raise RuntimeError when the neighbour ``nbr`` across ``side`` sizes the shared
    face differently. ``mine``/``theirs`` are ``(nxp, nyp, ngh)``; x-neighbours must
    agree on ``nyp`` and ngh, y-neighbours on ``nxp`` and ngh (mpi_halo.py:256-275): the
    extent across the face is the split axis and may differ."""
    (m_nxp, m_nyp, m_ngh), (t_nxp, t_nyp, t_ngh) = mine, theirs
    what, m, t = ("nyp", m_nyp, t_nyp) if side.startswith("x") else ("nxp", m_nxp, t_nxp)
    if m != t or m_ngh != t_ngh:
        raise RuntimeError(
            f"halo face {side}: rank {nbr} sizes this face differently -- local ({what}={m}, "
            f"ngh={m_ngh}), neighbour ({what}={t}, ngh={t_ngh}). Both ranks must pack the same "
            f"face: give them the same {what} and ngh (the extent across the face may differ).")


class Halo2D:
    """Persistent face exchanger for arrays of shape ``(*, nxp, W)``, ``W >= nyp``
    (the columns past ``nyp`` -- a row pitch -- are not touched).

    ``comm`` is a torch.distributed process group (None: the default group). Buffers
    are allocated on the first exchange of each leading shape, dtype and device, and
    reused."""

    def __init__(self, comm=None, nxp: int = 0, nyp: int = 0, ngh: int = 2,
                 dtype: str = "float64", periods=(False, False), dims=None,
                 device: Optional[torch.device] = None):
        if not dist.is_available() or not dist.is_initialized():
            raise RuntimeError("Halo2D needs an initialised torch.distributed process group")
        self.group = comm
        self.size = dist.get_world_size(comm)
        self.rank = dist.get_rank(comm)
        if dims is None:
            dims = compute_dims(self.size)
        else:
            dims = [int(d) for d in dims]
            if len(dims) != 2 or dims[0] < 1 or dims[1] < 1 or dims[0] * dims[1] != self.size:
                raise ValueError(f"dims {dims} mismatched with comm size {self.size}")
        self.dims = dims
        self.coords = (self.rank // dims[1], self.rank % dims[1])
        self.periods = (bool(periods[0]), bool(periods[1]))
        self.nxp, self.nyp, self.ngh = int(nxp), int(nyp), int(ngh)
        if self.ngh < 1 or self.nxp < 2 * self.ngh or self.nyp < 2 * self.ngh:
            raise ValueError(f"Halo2D: padded extent ({self.nxp}, {self.nyp}) too small for "
                             f"ngh={self.ngh}")
        self.dtype = str(dtype)
        self.backend = str(dist.get_backend(comm))
        # NCCL moves device buffers; every other backend goes through host memory
        self.device_direct = self.backend == "nccl"
        if device is None:
            device = (torch.device("cuda", torch.cuda.current_device()) if self.device_direct
                      else torch.device("cpu"))
        self.device = torch.device(device)
        cx, cy = self.coords
        self.nbr_x = (self._rank_at(cx - 1, cy), self._rank_at(cx + 1, cy))
        self.nbr_y = (self._rank_at(cx, cy - 1), self._rank_at(cx, cy + 1))
        self._bufs = {}
        self.exchanges = 0
        self._negotiate_face_extent()

    # ------------------------------------------------------------- topology
    def _rank_at(self, cx, cy):
        px, py = self.dims
        if not 0 <= cx < px:
            if not (self.periods[0] and px > 1):
                return None
            cx %= px
        if not 0 <= cy < py:
            if not (self.periods[1] and py > 1):
                return None
            cy %= py
        return cx * py + cy

    def _neighbor(self, side: str):
        return {"x-": self.nbr_x[0], "x+": self.nbr_x[1],
                "y-": self.nbr_y[0], "y+": self.nbr_y[1]}[side]

    def has_neighbor(self, side: str) -> bool:
        """True when the face ('x-', 'x+', 'y-', 'y+') borders another rank, False on a
        physical boundary."""
        return self._neighbor(side) is not None

    def _peer(self, group_rank):
        return group_rank if self.group is None else dist.get_global_rank(self.group, group_rank)

    def _comm_device(self):
        return self.device if self.device_direct else torch.device("cpu")

    def _negotiate_face_extent(self):
        """Every rank learns every rank's (nxp, nyp, ngh) first, then checks its own
        faces, so a mismatch raises on both ranks of the pair and no rank is left
        waiting inside the check (mpi_halo.py:361-387)."""
        mine = torch.tensor([self.nxp, self.nyp, self.ngh], dtype=torch.int64,
                            device=self._comm_device())
        every = [torch.empty_like(mine) for _ in range(self.size)]
        dist.all_gather(every, mine, group=self.group)
        for side in SIDES:
            nbr = self._neighbor(side)
            if nbr is not None:
                check_face_extent(side, nbr, (self.nxp, self.nyp, self.ngh),
                                  tuple(int(v) for v in every[nbr].tolist()))

    # ------------------------------------------------------------- buffers
    def _faces(self, arr):
        """(inner strip sent, ghost strip filled) per face, as views of ``arr``."""
        g, nxp, nyp = self.ngh, self.nxp, self.nyp
        a = arr[..., :nxp, :nyp]
        return {"x-": (a[..., g:2 * g, :], a[..., 0:g, :]),
                "x+": (a[..., nxp - 2 * g:nxp - g, :], a[..., nxp - g:nxp, :]),
                "y-": (a[..., :, g:2 * g], a[..., :, 0:g]),
                "y+": (a[..., :, nyp - 2 * g:nyp - g], a[..., :, nyp - g:nyp])}

    def _get_bufs(self, arr, faces):
        staged = arr.device.type != "cpu" and not self.device_direct
        key = (tuple(arr.shape[:-2]), arr.dtype, str(arr.device))
        if key not in self._bufs:
            dev = torch.device("cpu") if (staged or arr.device.type == "cpu") else arr.device
            pin = staged and torch.cuda.is_available()
            d = {}
            for side in SIDES:
                if self.has_neighbor(side):
                    shape = faces[side][0].shape
                    d[side] = (torch.empty(shape, dtype=arr.dtype, device=dev, pin_memory=pin),
                               torch.empty(shape, dtype=arr.dtype, device=dev, pin_memory=pin))
            self._bufs[key] = d
        return self._bufs[key]

    def _check(self, arr):
        if arr.dim() < 2 or arr.shape[-2] != self.nxp or arr.shape[-1] < self.nyp:
            raise ValueError(f"halo exchange expects (*, {self.nxp}, >={self.nyp}), got {tuple(arr.shape)}")
        if str(arr.dtype).replace("torch.", "") != self.dtype:
            raise ValueError(f"halo buffer dtype mismatch: configured for {self.dtype}, the array is "
                             f"{str(arr.dtype).replace('torch.', '')}")
        if self.device_direct and arr.device != self.device:
            raise ValueError(f"halo exchange over NCCL needs arrays on {self.device}, got {arr.device}")

    # ------------------------------------------------------------- exchange
    def start_exchange(self, arr):
        """Pack the inner strips and post the sends and receives; returns the handle
        for ``wait_exchange``. Work that reads no ghost cell may run in between."""
        self._check(arr)
        faces = self._faces(arr)
        bufs = self._get_bufs(arr, faces)
        sides = [s for s in SIDES if self.has_neighbor(s)]
        for s in sides:
            bufs[s][0].copy_(faces[s][0])
        works = self.post({s: bufs[s][0] for s in sides}, {s: bufs[s][1] for s in sides})
        self.exchanges += 1
        return {"works": works, "faces": faces, "bufs": bufs, "sides": sides}

    def post(self, sends, recvs):
        """Post one contiguous buffer to the neighbour across each side in ``sends`` and
        a receive from it into ``recvs[side]``; returns the works to wait on. The
        buffers are on the device for NCCL, in host memory otherwise."""
        ops = []
        # per axis: sends towards - then +, receives from + then -; so where both faces
        # of an axis border the same rank (two ranks on a periodic axis) the i-th message
        # between a pair lands in the i-th receive, with or without tags
        for lo, hi in (("x-", "x+"), ("y-", "y+")):
            for s in (lo, hi):
                if s in sends:
                    ops.append(dist.P2POp(dist.isend, sends[s], self._peer(self._neighbor(s)),
                                          self.group, _TAG[_OPPOSITE[s]]))
            for s in (hi, lo):
                if s in recvs:
                    ops.append(dist.P2POp(dist.irecv, recvs[s], self._peer(self._neighbor(s)),
                                          self.group, _TAG[s]))
        return dist.batch_isend_irecv(ops) if ops else []

    def wait_exchange(self, handle):
        """Complete the exchange: wait for the transfers, then unpack the received
        strips into the ghost cells."""
        for w in handle["works"]:
            w.wait()
        for s in handle["sides"]:
            handle["faces"][s][1].copy_(handle["bufs"][s][1])

    def exchange(self, arr):
        """Fill the ghost strips of ``arr`` that border another rank from that rank's
        inner strips; physical faces are left to the ghost fill."""
        self.wait_exchange(self.start_exchange(arr))

    # ------------------------------------------------------------- reductions
    def allreduce_max_(self, t):
        """In-place maximum over the ranks of a small tensor (the wave-speed bits)."""
        if t.device.type == "cpu" or self.device_direct:
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
            return t
        h = t.cpu()
        dist.all_reduce(h, op=dist.ReduceOp.MAX, group=self.group)
        t.copy_(h)
        return t

    def allreduce_min_(self, t):
        """In-place minimum over the ranks of a small tensor."""
        if t.device.type == "cpu" or self.device_direct:
            dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
            return t
        h = t.cpu()
        dist.all_reduce(h, op=dist.ReduceOp.MIN, group=self.group)
        t.copy_(h)
        return t

    def allreduce_sum_(self, t):
        """In-place sum over the ranks of a small tensor (the inlets' depth sums, float64,
        one batched collective for all inlets as the reference's Allreduce)."""
        if t.device.type == "cpu" or self.device_direct:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            return t
        h = t.cpu()
        dist.all_reduce(h, op=dist.ReduceOp.SUM, group=self.group)
        t.copy_(h)
        return t

    def check_same(self, value: int, what: str):
        """Raise on every rank unless every rank passes the same integer: a count that
        decides how many collectives a step posts (the number of discharge inlets)."""
        dev = self._comm_device()
        t = torch.tensor([int(value), -int(value)], dtype=torch.int64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        hi, lo = int(t[0]), -int(t[1])
        if hi != lo:
            raise RuntimeError(f"{what} differ across ranks (between {lo} and {hi}): pass the same list on "
                               f"every rank (entries may hold no local cells)")


class FlatHalo:
    """Seam exchange of the compressed mesh, the reference's ``CompressedHalo``
    (compressed_solver.py:1069-1132) on this package's brick slots.

    For each face that borders another rank, the stored cells of the ``ngh`` rows
    (columns) next to the face are gathered into a dense ``(3, ngh, P)`` buffer at
    ``(offset from the face's first row, position along the face)`` -- ``P = nyp`` for
    an x face, ``nxp`` for a y face -- and the neighbour scatters the positions of its
    own stored ghost cells out of it. Dense positions make the two ranks agree on the
    cell order whatever their stored sets are; a position the sender does not store
    arrives as 0, and only at a ghost cell that no active cell of the receiver reads.

    ``slot_pad`` is the ``(nxp, nyp)`` map of padded cell -> brick slot (-1 where not
    stored), ``nslots`` the length of the flat slot arrays exchanged. On the device one
    libgsw launch (``gsw_seam_copy``) packs or unpacks all three planes of a face; host
    planes (the CPU tests of this exchange) are indexed in place."""

    def __init__(self, halo: Halo2D, slot_pad, nslots: Optional[int] = None):
        self.halo = halo
        g, nxp, nyp = halo.ngh, halo.nxp, halo.nyp
        if tuple(slot_pad.shape) != (nxp, nyp):
            raise ValueError(f"FlatHalo: slot map {tuple(slot_pad.shape)} is not ({nxp}, {nyp})")
        dev = slot_pad.device
        top = int(slot_pad.max()) if slot_pad.numel() else -1
        if nslots is not None and top >= int(nslots):
            raise ValueError(f"FlatHalo: slot {top} outside the {int(nslots)} slots of the state")
        self.nslots = None if nslots is None else int(nslots)
        self.staged = not halo.device_direct and dev.type != "cpu"
        self.faces = {}
        for side in SIDES:
            if not halo.has_neighbor(side):
                continue
            if side[0] == "x":
                send = (slice(g, 2 * g) if side == "x-" else slice(nxp - 2 * g, nxp - g), slice(None))
                recv = (slice(0, g) if side == "x-" else slice(nxp - g, nxp), slice(None))
                sblk, rblk, P = slot_pad[send], slot_pad[recv], nyp
            else:
                send = (slice(None), slice(g, 2 * g) if side == "y-" else slice(nyp - 2 * g, nyp - g))
                recv = (slice(None), slice(0, g) if side == "y-" else slice(nyp - g, nyp))
                sblk, rblk, P = slot_pad[send].t(), slot_pad[recv].t(), nxp
            sflat, rflat = sblk.reshape(-1), rblk.reshape(-1)
            spos = torch.nonzero(sflat >= 0).reshape(-1)
            rpos = torch.nonzero(rflat >= 0).reshape(-1)
            f = dict(P=P, spos=spos, sslot=sflat[spos], rpos=rpos, rslot=rflat[rpos],
                     sdense=torch.zeros((3, g * P), dtype=torch.float32, device=dev),
                     rdense=torch.zeros((3, g * P), dtype=torch.float32, device=dev))
            if self.staged:
                pin = torch.cuda.is_available()
                f["shost"] = torch.zeros((3, g * P), dtype=torch.float32, pin_memory=pin)
                f["rhost"] = torch.zeros((3, g * P), dtype=torch.float32, pin_memory=pin)
            self.faces[side] = f
        self.exchanges = 0

    def send_cells(self, side):
        return int(self.faces[side]["spos"].numel()) if side in self.faces else 0

    @property
    def launches_per_exchange(self):
        """libgsw launches of one exchange of device planes (a pack and an unpack per face)."""
        return 2 * len(self.faces)

    def _seam(self, planes, slot, pos, dense, scatter):
        import ctypes as C
        from . import _lib as L
        if self.nslots is not None and planes[0].numel() != self.nslots:
            raise ValueError(f"FlatHalo: planes of {planes[0].numel()} slots, built for {self.nslots}")
        a = L.GswSeamArgs()
        a.abi_version = L.ABI_VERSION
        a.dtype = L.F32 if planes[0].dtype == torch.float32 else L.F64
        a.q0, a.q1, a.q2 = (C.c_void_p(p.data_ptr()) for p in planes)
        a.nslots = planes[0].numel()
        a.slot, a.pos = C.c_void_p(slot.data_ptr()), C.c_void_p(pos.data_ptr())
        a.n = slot.numel()
        a.dense, a.stride = C.c_void_p(dense.data_ptr()), dense.shape[1]
        a.scatter = int(scatter)
        L.call("gsw_seam_copy", C.byref(a), C.c_void_p(torch.cuda.current_stream().cuda_stream))

    def exchange(self, planes):
        """Refresh the stored seam ghost cells of the three flat planes in place."""
        self.finish(self.start(planes))

    def start(self, planes):
        """Pack the seam cells of the three flat planes and post the sends and receives;
        returns the handle for ``finish``. Work that reads and writes no seam ghost cell
        of ``planes`` may run in between (over NCCL, on the device while the transfer is
        in flight)."""
        device = planes[0].device.type != "cpu"
        if any(p.dtype != torch.float32 for p in planes):
            raise ValueError("FlatHalo: the compressed state is float32")
        sends, recvs = {}, {}
        for side, f in self.faces.items():
            if device:
                self._seam(planes, f["sslot"], f["spos"], f["sdense"], 0)
            else:
                for c in range(3):
                    f["sdense"][c].index_copy_(0, f["spos"], planes[c].index_select(0, f["sslot"]))
            if self.staged:
                f["shost"].copy_(f["sdense"])
                sends[side], recvs[side] = f["shost"], f["rhost"]
            else:
                sends[side], recvs[side] = f["sdense"], f["rdense"]
        return {"planes": planes, "device": device, "works": self.halo.post(sends, recvs)}

    def finish(self, handle):
        """Wait for the transfers of ``start`` and scatter the received seam cells into
        the stored ghost slots."""
        planes, device = handle["planes"], handle["device"]
        for w in handle["works"]:
            w.wait()
        for side, f in self.faces.items():
            if self.staged:
                f["rdense"].copy_(f["rhost"])
            if device:
                self._seam(planes, f["rslot"], f["rpos"], f["rdense"], 1)
            else:
                for c in range(3):
                    planes[c].index_copy_(0, f["rslot"], f["rdense"][c].index_select(0, f["rpos"]))
        self.exchanges += 1
