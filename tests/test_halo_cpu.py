"""The Cartesian split of the dense grid on the CPU: the strip bounds (pinned to the
reference's own partition tests, tests/test_partition.py), the face exchange of
``halo.Halo2D`` between gloo ranks, and a split oracle run -- each rank the oracle's
NumPy step on its block, ghosts at the seams from ``Halo2D``, dt the minimum over the
ranks -- equal bit for bit to the single-domain oracle run. The oracle is the
checker; the exchange under test is the package's."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from geoswe_b200.halo import SIDES, Halo2D, check_face_extent, compute_dims  # noqa: E402
from geoswe_b200.partition import block_of, strip_bounds  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(fn, world, *args):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(fn, args=(world, _free_port(), out, *args), nprocs=world,
                           start_method="spawn", join=True)
        return dict(out)


def _init(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)


# ------------------------------------------------------------------ layout
def test_compute_dims_is_the_most_square_split():
    want = {1: [1, 1], 2: [2, 1], 3: [3, 1], 4: [2, 2], 6: [3, 2], 7: [7, 1], 8: [4, 2],
            12: [4, 3], 16: [4, 4]}
    assert {n: compute_dims(n) for n in want} == want


def test_strip_bounds_pins():
    """Known answers of the reference's tests/test_partition.py."""
    assert strip_bounds(32000 * 16, 16) == [32000 * r for r in range(17)]
    assert strip_bounds(10, 3) == [0, 3, 7, 10]
    assert strip_bounds(7, 1) == [0, 7]
    for n, k in ((4096, 4), (1000, 7), (33, 5)):
        w = np.linspace(0.97, 1.03, k)
        assert strip_bounds(n, k, w) == strip_bounds(np.ones(n), k, w)
    rng = np.random.default_rng(0)
    w = 1.0 + 0.0056 * rng.standard_normal(1024)
    n = 32000 * w.size
    jb = strip_bounds(n, w.size, w)
    strips = np.diff(jb)
    assert jb[0] == 0 and jb[-1] == n and (strips > 0).all()
    assert np.abs(strips - n * w / w.sum()).max() <= 1.0
    col = np.r_[np.zeros(100), np.full(300, 5.0), np.full(600, 1.0)]
    jb = strip_bounds(col, 3, [1.0, 1.0, 1.0])
    assert max(abs(col[jb[r]:jb[r + 1]].sum() - 700.0) for r in range(3)) <= 5.0
    jb = strip_bounds(col, 2, [3.0, 1.0])
    assert abs(col[:jb[1]].sum() - 0.75 * col.sum()) <= 5.0
    assert strip_bounds(4, 4, [1e-9, 1.0, 1.0, 1e-9]) == [0, 1, 2, 3, 4]
    jb = strip_bounds(np.r_[np.zeros(50), 1.0, np.zeros(49)], 3)
    assert jb[0] == 0 and jb[-1] == 100 and all(b > a for a, b in zip(jb, jb[1:]))


@pytest.mark.parametrize("bad", [[1.0, 1.0], [1.0, 0.0, 1.0], [1.0, -1.0, 1.0], [1.0, np.nan, 1.0],
                                 [1.0, np.inf, 1.0]])
def test_strip_bounds_refuses_bad_weights(bad):
    with pytest.raises(ValueError, match="weights"):
        strip_bounds(300, 3, bad)


def test_strip_bounds_refuses_too_many_ranks():
    with pytest.raises(ValueError, match="cannot be split"):
        strip_bounds(3, 4)
    with pytest.raises(ValueError, match="n_ranks"):
        strip_bounds(3, 0)


def test_blocks_tile_the_grid():
    nx, ny, dims = 23, 18, (3, 2)
    cover = np.zeros((nx, ny), int)
    for r in range(6):
        x0, x1, y0, y1 = block_of(nx, ny, dims, (r // 2, r % 2))
        cover[x0:x1, y0:y1] += 1
    assert (cover == 1).all()


def test_members_split_by_work():
    from geoswe_b200.partition import members_of
    work = [100] * 48 + [400] * 16                  # 64 members, the last 16 four times larger
    parts = [members_of(work, 4, r) for r in range(4)]
    assert [p.start for p in parts] == [0, 28, 50, 57] and parts[-1].stop == 64
    assert [sum(work[i] for i in p) for p in parts] == [2800] * 4
    assert list(members_of(64, 8, 3)) == list(range(24, 32))
    with pytest.raises(ValueError, match="rank"):
        members_of(64, 8, 8)


def test_face_extent_message():
    """Mirrors the reference's check (mpi_halo.py:256-275): only the extent along the
    face must agree, and the message names the face, the rank and both extents."""
    mine = (40, 24, 4)
    for side, nbr, theirs, want in (("x-", 3, (40, 20, 4), ("face x-", "rank 3", "nyp=24", "nyp=20")),
                                    ("y+", 1, (36, 24, 4), ("face y+", "nxp=40", "nxp=36")),
                                    ("x+", 1, (40, 24, 2), ("ngh=4", "ngh=2"))):
        with pytest.raises(RuntimeError) as e:
            check_face_extent(side, nbr, mine, theirs)
        assert all(w in str(e.value) for w in want), str(e.value)
    for side, theirs in (("x-", (33, 24, 4)), ("x+", (33, 24, 4)), ("y-", (40, 19, 4)), ("y+", (40, 19, 4))):
        check_face_extent(side, 1, mine, theirs)


# ------------------------------------------------------------------ exchange
NX, NY, G = 23, 18, 2


def _exchange_rank(rank, world, port, out, dims, periods):
    _init(rank, world, port)
    try:
        cx, cy = rank // dims[1], rank % dims[1]
        x0, x1, y0, y1 = block_of(NX, NY, dims, (cx, cy))
        nx, ny = x1 - x0, y1 - y0
        halo = Halo2D(None, nx + 2 * G, ny + 2 * G, G, dtype="float64", periods=periods, dims=dims)
        W = ny + 2 * G + 3                            # a row pitch past nyp stays untouched
        a = torch.full((3, nx + 2 * G, W), -1.0, dtype=torch.float64)
        gi = torch.arange(x0, x1, dtype=torch.float64)[:, None]
        gj = torch.arange(y0, y1, dtype=torch.float64)[None, :]
        for c in range(3):
            a[c, G:G + nx, G:G + ny] = c * 1e6 + gi * 1000 + gj
        halo.exchange(a)
        bad = []
        for i in range(nx + 2 * G):
            for j in range(W):
                inner_i, inner_j = G <= i < G + nx, G <= j < G + ny
                if inner_i and inner_j:
                    continue
                got = a[:, i, j]
                if j >= ny + 2 * G or not (inner_i or inner_j):   # pitch columns, corners
                    if j >= ny + 2 * G and (got != -1.0).any():
                        bad.append(("pitch", i, j))
                    continue
                side = ("x-" if i < G else "x+") if not inner_i else ("y-" if j < G else "y+")
                if not halo.has_neighbor(side):
                    if (got != -1.0).any():
                        bad.append(("physical face written", side, i, j))
                    continue
                ii, jj = x0 + i - G, y0 + j - G
                ii, jj = ii % NX, jj % NY
                want = torch.tensor([c * 1e6 + ii * 1000 + jj for c in range(3)], dtype=torch.float64)
                if not torch.equal(got, want):
                    bad.append((side, i, j, got.tolist(), want.tolist()))
        out[rank] = dict(bad=bad[:5], nbad=len(bad), nbr=(halo.nbr_x, halo.nbr_y),
                         sides=[s for s in SIDES if halo.has_neighbor(s)])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims,periods", [
    (2, [2, 1], (False, False)),
    (2, [1, 2], (False, False)),
    (2, [2, 1], (True, False)),          # both x faces border the same rank
    (2, [2, 1], (False, True)),          # periodic y not split: the ghost fill's wrap
    (4, [2, 2], (True, True)),
    (4, [4, 1], (False, False)),
])
def test_exchange_fills_seams_only(world, dims, periods):
    out = _spawn(_exchange_rank, world, dims, periods)
    for r in range(world):
        assert out[r]["nbad"] == 0, (r, out[r])
    if dims == [2, 1] and periods == (True, False):
        assert out[0]["nbr"][0] == (1, 1) and set(out[0]["sides"]) == {"x-", "x+"}
    if periods == (False, True):
        assert all("y-" not in out[r]["sides"] for r in range(world))


def _mismatch_rank(rank, world, port, out):
    _init(rank, world, port)
    try:
        Halo2D(None, 20, 10 + 2 * rank, G, dtype="float32", dims=[2, 1])
        out[rank] = "accepted"
    except RuntimeError as e:
        out[rank] = str(e)
    finally:
        dist.destroy_process_group()


def test_face_extent_mismatch_raises_on_both_ranks():
    out = _spawn(_mismatch_rank, 2)
    assert "nyp=10" in out[0] and "nyp=12" in out[0] and "rank 1" in out[0]
    assert "nyp=12" in out[1] and "nyp=10" in out[1] and "rank 0" in out[1]


def _inlet_count_rank(rank, world, port, out):
    _init(rank, world, port)
    try:
        h = Halo2D(None, 20, 10, G, dtype="float32", dims=[world, 1])
        sums = torch.tensor([1.5 * (rank + 1), 0.0 if rank else 2.25], dtype=torch.float64)
        h.allreduce_sum_(sums)
        h.check_same(2, "inlets")                       # every rank lists two inlets
        res = [float(x) for x in sums]
        try:
            h.check_same(2 + rank, "inlets")            # rank 1 lists one more
            res.append("accepted")
        except RuntimeError as e:
            res.append(str(e))
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_inlet_sums_and_counts_over_ranks():
    """The per-inlet depth sums of a split run are added over the ranks in one collective,
    and a rank listing a different number of inlets (so a different number of
    collectives per step) is refused on every rank instead of hanging."""
    out = _spawn(_inlet_count_rank, 2)
    for r in range(2):
        assert out[r][:2] == [1.5 + 3.0, 2.25]
        assert "differ across ranks" in out[r][2] and "between 2 and 3" in out[r][2]


def _dry_bed(k, rank):
    """Inlet k's bed values on `rank` (inlet 1 has no cells on rank 1; inlet 2 is flat)."""
    rng = np.random.default_rng(100 * k + rank)
    if k == 1 and rank == 1:
        return np.zeros(0, np.float32)
    if k == 2:
        return np.full(3 + rank, 7.25, np.float32)
    return (5.0 + rng.random(4 + 3 * rank) * 2.0).astype(np.float32)


def _dry_seed_local(z):
    """The single-domain kernel's dry seed reductions over all of an inlet's cells."""
    zmin, zmax = float(z.min()), float(z.max())
    seed = np.float32(zmin + 0.10 * (zmax - zmin))
    return zmin, zmax, float(np.count_nonzero(z <= np.float32(zmin))), float(np.maximum(seed - z, 0).max())


def _dry_seed_rank(rank, world, port, out):
    _init(rank, world, port)
    try:
        from geoswe_b200.compressed import inlet_dry_reductions
        h = Halo2D(None, 20, 10, G, dtype="float32", dims=[world, 1])
        out[rank] = inlet_dry_reductions([_dry_bed(k, rank) for k in range(3)], h, torch.device("cpu"))
    finally:
        dist.destroy_process_group()


def test_inlet_dry_seed_reductions_over_ranks():
    """A dry inlet's seed (bed range, cells at the minimum, largest seed depth) is reduced
    over every rank's cells, as the reference does once at setup: two ranks give the
    values the single-domain kernel computes from all the cells, including an inlet
    with no cells on one rank and a flat one."""
    out = _spawn(_dry_seed_rank, 2)
    for k in range(3):
        want = _dry_seed_local(np.concatenate([_dry_bed(k, r) for r in range(2)]))
        for r in range(2):
            assert out[r][k] == want, (k, r, out[r][k], want)
    assert out[0][2][3] == 0.0                     # the flat inlet: no seed depth anywhere


def _placement_rank(rank, world, port, out, dims, nx, ny):
    _init(rank, world, port)
    try:
        from geoswe_b200.compressed import CompressedSolver
        x0, x1, y0, y1 = block_of(nx, ny, dims, (rank // dims[1], rank % dims[1]))
        cs = CompressedSolver()
        cs.halo = Halo2D(None, x1 - x0 + 4, y1 - y0 + 4, 2, dtype="float32", dims=dims)
        cs.nx, cs.ny = x1 - x0, y1 - y0
        out[rank] = (cs._placement(), (x0, y0))
    finally:
        dist.destroy_process_group()


def test_split_cache_placement():
    """A split cache records each block's place in the global grid (the reference's
    `placement` and global extents), gathered from every rank's block extents: uneven
    blocks of a 2 x 2 split land at the offsets `partition.block_of` gave them."""
    out = _spawn(_placement_rank, 4, [2, 2], 37, 53)
    for r in range(4):
        (pl, glob), (x0, y0) = out[r]
        assert (pl["i0"], pl["j0"]) == (x0, y0) and glob == (37, 53), (r, pl, glob)


# ------------------------------------------------------------------ split oracle run
NSTEPS = 25


def _oracle_inputs(dtype):
    from tests._cases import flowing
    return flowing(NX, NY, seed=5, dtype=dtype)


def _oracle_solver(qp, bp, kinds, dtype):
    from oracle.numpy_ref import NumpySolver2D
    return NumpySolver2D(qp, bp, G, 2.0, 2.5, kinds=kinds, friction="manning", manning_n=0.03,
                         rain_times=[0.0, 1e9], rain_mm_h=[80.0, 80.0])


def _kinds_axes(kinds):
    return ("periodic" if kinds[0] == "periodic" else "x", "periodic" if kinds[2] == "periodic" else "y")


def _split_rank(rank, world, port, out, dims, kinds, dtype):
    _init(rank, world, port)
    try:
        from geoswe_b200.solver import pad_bed
        dtype = np.dtype(dtype)
        q0, bed = _oracle_inputs(dtype)
        periods = (kinds[0] == "periodic", kinds[2] == "periodic")
        coords = (rank // dims[1], rank % dims[1])
        x0, x1, y0, y1 = block_of(NX, NY, dims, coords)
        nx, ny = x1 - x0, y1 - y0
        halo = Halo2D(None, nx + 2 * G, ny + 2 * G, G, dtype=str(dtype), periods=periods, dims=dims)
        qp = np.zeros((3, nx + 2 * G, ny + 2 * G), dtype)
        qp[:, G:G + nx, G:G + ny] = q0[:, x0:x1, y0:y1]
        bp = np.zeros((nx + 2 * G, ny + 2 * G), dtype)
        bp[G:G + nx, G:G + ny] = bed[x0:x1, y0:y1]
        bx, by = _kinds_axes(kinds)
        pad_bed(bp, G, bx, by)
        halo.exchange(torch.from_numpy(bp))
        local = [("none" if halo.has_neighbor(s) else k) for s, k in zip(SIDES, kinds)]
        s = _oracle_solver(qp, bp, local, dtype)
        dts = []
        for _ in range(NSTEPS):
            dt = s.rain_step_limit(s.cfl_dt())
            dt = float(halo.allreduce_min_(torch.tensor([dt], dtype=torch.float64))[0])
            halo.exchange(torch.from_numpy(s.q))
            s.step(dt)
            dts.append(dt)
        out[rank] = dict(block=(x0, x1, y0, y1), q=s.q[:, G:G + nx, G:G + ny].copy(),
                         bed=bp.copy(), dts=dts)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims,kinds,dtype", [
    (2, [2, 1], ("wall", "fall", "wall", "wall"), "float32"),
    (2, [1, 2], ("wall", "fall", "extrapolate", "wall"), "float32"),
    (2, [2, 1], ("periodic", "periodic", "wall", "wall"), "float64"),
    (4, [2, 2], ("periodic",) * 4, "float32"),
    (3, [1, 3], ("fall", "wall", "wall", "fall"), "float64"),
])
def test_split_oracle_run_equals_single_domain(world, dims, kinds, dtype):
    from geoswe_b200.solver import pad_bed
    out = _spawn(_split_rank, world, dims, kinds, dtype)
    dt_ = np.dtype(dtype)
    q0, bed = _oracle_inputs(dt_)
    qp = np.zeros((3, NX + 2 * G, NY + 2 * G), dt_)
    qp[:, G:-G, G:-G] = q0
    bp = np.zeros((NX + 2 * G, NY + 2 * G), dt_)
    bp[G:-G, G:-G] = bed
    bx, by = _kinds_axes(kinds)
    pad_bed(bp, G, bx, by)
    s = _oracle_solver(qp, bp, list(kinds), dt_)
    dts = []
    for _ in range(NSTEPS):
        dt = s.rain_step_limit(s.cfl_dt())
        s.step(dt)
        dts.append(dt)
    for r in range(world):
        x0, x1, y0, y1 = out[r]["block"]
        assert out[r]["dts"] == dts, r
        np.testing.assert_array_equal(out[r]["q"], s.q[:, G + x0:G + x1, G + y0:G + y1])
        # the exchanged bed equals the single-domain padded bed away from the corners
        lb = out[r]["bed"]
        gb = bp[x0:x1 + 2 * G, y0:y1 + 2 * G]
        if x0 == 0 and bx == "periodic":
            gb = None                     # the wrap's image lies at the far end; checked by q
        if gb is not None and y0 == 0 and by == "periodic":
            gb = None
        if gb is not None and x1 == NX and bx == "periodic":
            gb = None
        if gb is not None and y1 == NY and by == "periodic":
            gb = None
        if gb is not None:
            np.testing.assert_array_equal(lb[G:-G, :], gb[G:-G, :])
            np.testing.assert_array_equal(lb[:, G:-G], gb[:, G:-G])
    assert s.q[0, G:-G, G:-G].max() > 0.5           # a flowing case, not a trivial one


# ------------------------------------------------------------------ compressed-mesh seams
def _flat_rank(rank, world, port, out, dims):
    _init(rank, world, port)
    try:
        from geoswe_b200.halo import FlatHalo
        rng = np.random.default_rng(11)
        glob = rng.random((NX + 2 * G, NY + 2 * G)) < 0.7          # stored cells, global padded frame
        cx, cy = rank // dims[1], rank % dims[1]
        x0, x1, y0, y1 = block_of(NX, NY, dims, (cx, cy))
        nxp, nyp = x1 - x0 + 2 * G, y1 - y0 + 2 * G
        halo = Halo2D(None, nxp, nyp, G, dtype="float32", dims=dims)
        stored = glob[x0:x0 + nxp, y0:y0 + nyp].copy()
        ghost = np.ones((nxp, nyp), bool)
        ghost[G:-G, G:-G] = False
        extra = ghost & ~stored & (np.random.default_rng(100 + rank).random((nxp, nyp)) < 0.3)
        stored |= extra                                              # ghosts the owner does not store
        n = int(stored.sum())
        slots = np.random.default_rng(200 + rank).permutation(n + 5)[:n]
        slot_pad = np.full((nxp, nyp), -1, np.int64)
        slot_pad[stored] = slots
        planes = [torch.full((n + 5,), -1.0) for _ in range(3)]
        ii, jj = np.nonzero(stored & ~ghost)
        for c in range(3):
            planes[c][torch.from_numpy(slot_pad[ii, jj])] = torch.from_numpy(
                (c * 1e6 + (x0 + ii - G) * 1000 + (y0 + jj - G)).astype(np.float32))
        fh = FlatHalo(halo, torch.from_numpy(slot_pad))
        fh.exchange(planes)
        bad = []
        for i, j in zip(*np.nonzero(stored)):
            got = [float(planes[c][slot_pad[i, j]]) for c in range(3)]
            inner_i, inner_j = G <= i < nxp - G, G <= j < nyp - G
            if inner_i and inner_j:
                want = [c * 1e6 + (x0 + i - G) * 1000 + (y0 + j - G) for c in range(3)]
            elif not (inner_i or inner_j):
                continue     # corners: a y face spans the full x extent, as the reference's does
            else:
                side = ("x-" if i < G else "x+") if not inner_i else ("y-" if j < G else "y+")
                if not halo.has_neighbor(side):
                    want = [-1.0] * 3
                elif extra[i, j]:
                    want = [0.0] * 3                                 # the sender stores no such cell
                else:
                    want = [c * 1e6 + (x0 + i - G) * 1000 + (y0 + j - G) for c in range(3)]
            if got != want:
                bad.append((int(i), int(j), got, want))
        untouched = all(float(planes[c][s]) == -1.0 for c in range(3)
                        for s in sorted(set(range(n + 5)) - set(slots.tolist())))
        out[rank] = dict(nbad=len(bad), bad=bad[:4], untouched=untouched,
                         sent=sum(fh.send_cells(s) for s in SIDES))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims", [(2, [2, 1]), (2, [1, 2]), (4, [2, 2])])
def test_flat_seam_exchange(world, dims):
    out = _spawn(_flat_rank, world, dims)
    for r in range(world):
        assert out[r]["nbad"] == 0, (r, out[r]["bad"])
        assert out[r]["untouched"] and out[r]["sent"] > 0


def test_comm_must_be_a_process_group():
    from geoswe_b200.halo import comm_size
    assert comm_size(None) == 1

    class MpiLike:
        size, rank = 4, 0
    with pytest.raises(TypeError, match="ProcessGroup"):
        comm_size(MpiLike())


# ------------------------------------------------------------------ split compressed oracle run
CX, CY, CSTEPS = 40, 34, 30


def _flat_global():
    from tests._cases import flowing
    from geoswe_b200.solver import pad_bed
    from geoswe_b200.synthetic import dilate_cross
    q0, bed = flowing(CX, CY, seed=21, dtype=np.float32)
    rng = np.random.default_rng(21)
    m = np.zeros((CX, CY), bool)
    m[rng.integers(3, CX - 3, 7), rng.integers(3, CY - 3, 7)] = True
    m = dilate_cross(m, 6)
    m[:2, :] = m[-2:, :] = False
    m[:, :2] = m[:, -2:] = False
    qp = np.zeros((3, CX + 2 * G, CY + 2 * G), np.float32)
    qp[:, G:-G, G:-G] = q0 * m
    bp = np.zeros((CX + 2 * G, CY + 2 * G), np.float32)
    bp[G:-G, G:-G] = bed
    pad_bed(bp, G, "fall", "fall")
    inside = np.zeros((CX + 2 * G, CY + 2 * G), np.uint8)
    inside[G:-G, G:-G] = m
    return qp, bp, inside


def _flat_oracle(tab, act, qp, bp):
    import oracle
    ij = tab["ij"]
    return oracle.OracleFlat(tab["nbr"], act, [qp[c][ij[:, 0], ij[:, 1]] for c in range(3)],
                             bp[ij[:, 0], ij[:, 1]], 2.0, ntab=(0.03,), rain_times=[0.0, 1e9],
                             rain_table=np.full((2, 1), 90.0 / 3.6e6, np.float32),
                             rain_lookup=np.zeros(len(act), np.int64))


def _flat_split_rank(rank, world, port, out, dims):
    _init(rank, world, port)
    try:
        from geoswe_b200.compressed import build_tables
        from geoswe_b200.halo import FlatHalo
        qp, bp, inside_g = _flat_global()
        x0, x1, y0, y1 = block_of(CX, CY, dims, (rank // dims[1], rank % dims[1]))
        nxp, nyp = x1 - x0 + 2 * G, y1 - y0 + 2 * G
        halo = Halo2D(None, nxp, nyp, G, dtype="float32", dims=dims)
        own = np.zeros((nxp, nyp), np.uint8)
        own[G:-G, G:-G] = inside_g[x0 + G:x1 + G, y0 + G:y1 + G]
        ext = torch.from_numpy(own.astype(np.float32))
        halo.exchange(ext)                       # the neighbours' inside cells in the seam rows
        tab = build_tables((ext.numpy() > 0.5).astype(np.uint8), ring=2)
        ij = tab["ij"]
        act = own[ij[:, 0], ij[:, 1]]
        o = _flat_oracle(tab, act, qp[:, x0:x0 + nxp, y0:y0 + nyp], bp[x0:x0 + nxp, y0:y0 + nyp])
        slot_pad = np.full((nxp, nyp), -1, np.int64)
        slot_pad[ij[:, 0], ij[:, 1]] = np.arange(len(ij))
        fh = FlatHalo(halo, torch.from_numpy(slot_pad), nslots=len(ij))
        dts = []
        for _ in range(CSTEPS):
            lam = o._lammax() if o._lam is None else o._lam
            lam = float(halo.allreduce_max_(torch.tensor([lam], dtype=torch.float64))[0])
            dt = o.dt_from_lam(lam)
            fh.exchange([torch.from_numpy(x) for x in o.q])
            o.step(dt)
            dts.append(dt)
        keep = act != 0
        out[rank] = dict(ij=(ij[keep] + [x0, y0]).tolist(), h=o.q[0][keep].tolist(), dts=dts,
                         seam=sum(fh.send_cells(s) for s in SIDES))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims", [(2, [2, 1]), (2, [1, 2]), (4, [2, 2])])
def test_split_flat_oracle_run_equals_single_domain(world, dims):
    """The compressed split's design on the flat oracle: per rank the stored set grows
    from its own inside cells plus the neighbours' in the seam ghost rows, only its own
    cells are active, the seam cells come through FlatHalo before every step and the
    wave speed is the maximum over the ranks. The active cells equal the single-domain
    flat oracle run bit for bit."""
    from geoswe_b200.compressed import build_tables
    out = _spawn(_flat_split_rank, world, dims)
    qp, bp, inside_g = _flat_global()
    tab = build_tables(inside_g, ring=2)
    o = _flat_oracle(tab, tab["is_active"], qp, bp)
    dts = []
    for _ in range(CSTEPS):
        lam = o._lammax() if o._lam is None else o._lam
        dt = o.dt_from_lam(lam)
        o.step(dt)
        dts.append(dt)
    at = {tuple(p): k for k, p in enumerate(tab["ij"].tolist())}
    seen = 0
    for r in range(world):
        assert out[r]["dts"] == dts, r
        assert out[r]["seam"] > 0
        for p, h in zip(out[r]["ij"], out[r]["h"]):
            assert np.float32(h) == o.q[0][at[tuple(p)]], (r, p)
        seen += len(out[r]["h"])
    assert seen == int(tab["is_active"].sum())
    assert float(o.q[0][tab["is_active"] != 0].max()) > 0.1


@pytest.mark.parametrize("seams", [("x-",), ("x+", "y-"), ("x-", "x+", "y-", "y+")])
def test_seam_bricks_ordered_last(seams):
    """A split compressed run orders the bricks that read a seam ghost strip last: the
    bricks before them have no cell within 3 rows or columns of a seam strip (the step
    reads 2), the brick set and the neighbour links are those of the unsplit layout, and
    Hilbert order is kept within each part."""
    from geoswe_b200.compressed import BRICK_W, CompressedSolver
    rng = np.random.default_rng(3)
    nxp, nyp, g = 83, 131, 2
    inside = torch.from_numpy((rng.random((nxp, nyp)) < 0.7).astype(np.uint8))
    inside[:g], inside[-g:], inside[:, :g], inside[:, -g:] = 0, 0, 0, 0

    def layout(seams):
        cs = CompressedSolver()
        cs._init_physics(device="cpu", nxp=nxp, nyp=nyp, ngh=g, nx=nxp - 2 * g, ny=nyp - 2 * g, dx=1.0, g=9.81,
                         cfl=0.5, h_min=1e-6, cfl_linf=False, vcap=1.0, quad=True, keep_h=True, dt_max=None,
                         brick_h=8)
        cs._build_layout(inside, seams=seams)
        return cs, cs._bij.numpy().astype(np.int64), cs._bnbr.numpy().astype(np.int64)

    plain, pij, pnbr = layout(())
    cs, bij, bnbr = layout(seams)
    nb, ni, bh = cs.n_bricks, cs.n_bricks_inner, cs.brick_h
    assert nb == plain.n_bricks and plain.n_bricks_inner == nb and 0 < ni < nb
    key = lambda ij: [tuple(x) for x in ij]
    assert sorted(key(bij)) == sorted(key(pij))
    pos = {k: n for n, k in enumerate(key(pij))}
    # each part keeps the unsplit (Hilbert) order
    for part in (bij[:ni], bij[ni:]):
        order = [pos[k] for k in key(part)]
        assert order == sorted(order)
    # neighbour links point at the same bricks; missing neighbours stay the zero brick
    for b in range(nb):
        pb = pos[tuple(bij[b])]
        for d in range(4):
            want = pnbr[pb, d]
            got = bnbr[b, d]
            assert (got == nb) == (want == nb)
            if got != nb:
                assert tuple(bij[got]) == tuple(pij[want])
    # inner bricks are at least 3 cells from every seam strip
    r0, c0 = bij[:ni, 0] * bh, bij[:ni, 1] * BRICK_W
    if "x-" in seams:
        assert (r0 >= g + 3).all()
    if "x+" in seams:
        assert (r0 + bh - 1 < nxp - g - 3).all()
    if "y-" in seams:
        assert (c0 >= g + 3).all()
    if "y+" in seams:
        assert (c0 + BRICK_W - 1 < nyp - g - 3).all()
