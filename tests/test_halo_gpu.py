"""A dense run split over ranks equals the single-domain run bit for bit.

Two (or, for a 2 x 2 split, four) processes share the one GPU, each a rank of a gloo
group running ``Solver2D`` on its block (faces staged through host memory, as the exchange does for any backend but
NCCL); the kernels of the two processes never wait on each other -- every wait is on
the host, in the gloo calls. The single-domain run is this process's own.
"""
import os
import socket

import numpy as np
import pytest

from tests._cases import flowing

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

NX, NY, T_END = 46, 37, 6.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _make(mesh_shape, bc, dtype, q0, bed, **kw):
    from geoswe_b200 import Config, Mesh2D, Solver2D
    mesh = Mesh2D(nx=mesh_shape[0], ny=mesh_shape[1], dx=2.0, dy=2.5, ngh=2)
    cfg = Config(bc_x=bc[0], bc_y=bc[1], dtype=dtype, friction="manning", manning_n=0.03,
                 rainfall=80.0 / 3.6e6)
    return Solver2D(mesh, cfg, q0, bed, **kw)


def _rank(rank, world, port, out, dims, bc, dtype, host_loop):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from geoswe_b200.partition import block_of
        q0, bed = flowing(NX, NY, seed=5, dtype=np.dtype(dtype))
        x0, x1, y0, y1 = block_of(NX, NY, dims, (rank // dims[1], rank % dims[1]))
        s = _make((x1 - x0, y1 - y0), bc, dtype, q0[:, x0:x1, y0:y1].copy(), bed[x0:x1, y0:y1].copy(),
                  comm=dist.group.WORLD, dims=dims)
        if host_loop:
            steps = s.run(T_END, callback=lambda solver, k: None)
        else:
            steps = s.run(T_END)
        q = s.q_interior.detach().cpu().numpy().copy()
        out[rank] = dict(block=(x0, x1, y0, y1), steps=steps, t=s.t, q=q,
                         exchanges=s.halo.exchanges, launches=s.kernel_launches)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dims,bc,dtype,host_loop", [
    ([2, 1], ("wall", "extrapolate"), "float32", False),
    ([1, 2], ("wall", "wall"), "float32", False),
    ([2, 1], ("periodic", "wall"), "float64", True),
    # four bands around the interior window, the y-bands limited to the rows between the x-bands
    ([2, 2], ("wall", "extrapolate"), "float32", False),
])
def test_split_run_equals_single_domain(dims, bc, dtype, host_loop):
    q0, bed = flowing(NX, NY, seed=5, dtype=np.dtype(dtype))
    ref = _make((NX, NY), bc, dtype, q0, bed)
    ref_steps = ref.run(T_END, callback=(lambda solver, k: None) if host_loop else None)
    want = ref.q_interior.detach().cpu().numpy()
    torch.cuda.synchronize()
    world = dims[0] * dims[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out, dims, bc, dtype, host_loop), nprocs=world,
                           start_method="spawn", join=True)
        out = dict(out)
    assert ref_steps > 20
    for r in range(world):
        o = out[r]
        x0, x1, y0, y1 = o["block"]
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps, o["t"], ref.t)
        assert o["exchanges"] >= ref_steps and o["launches"] > 0
        np.testing.assert_array_equal(o["q"], want[:, x0:x1, y0:y1])


# Two discharge inlets (global padded indices, inward normal, hydrograph): one on the x-
# face, inside rank 0's block; one on the y- face, across the x seam of a [2, 1] split.
INLETS = [(np.full(6, 2), np.arange(6, 12), (1.0, 0.0), [0.0, 3.0, 6.0], [0.0, 4.0, 1.0]),
          (np.arange(12, 34), np.full(22, 2), (0.0, 1.0), [0.0, 6.0], [2.0, 0.5])]


def _add_inlets(s, block):
    """The inlets' cells inside `block` (unpadded [x0, x1) x [y0, y1)), in local padded
    indices; an inlet with no cells here is added empty, as every rank must list it."""
    x0, x1, y0, y1 = block
    for ii, jj, nrm, tq, q in INLETS:
        keep = (ii - 2 >= x0) & (ii - 2 < x1) & (jj - 2 >= y0) & (jj - 2 < y1)
        s.add_inflow(ii[keep] - x0, jj[keep] - y0, nrm, 2.0, tq, q)


def _inlet_rank(rank, world, port, out, dims):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from geoswe_b200.partition import block_of
        q0, bed = flowing(NX, NY, seed=5, dtype=np.float32)
        blk = block_of(NX, NY, dims, (rank // dims[1], rank % dims[1]))
        x0, x1, y0, y1 = blk
        s = _make((x1 - x0, y1 - y0), ("wall", "wall"), "float32", q0[:, x0:x1, y0:y1].copy(),
                  bed[x0:x1, y0:y1].copy(), comm=dist.group.WORLD, dims=dims)
        _add_inlets(s, blk)
        steps = s.run(T_END)
        out[rank] = dict(block=blk, steps=steps, t=s.t, q=s.q_interior.detach().cpu().numpy().copy())
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dims", [[1, 2], [2, 1]])
def test_split_run_with_inlets(dims):
    """Discharge inlets on a split run: each rank's share of an inlet's depth is summed
    over the ranks every step (the reference's batched Allreduce). An inlet within one
    rank gives the single-domain run bit for bit ([1, 2]: both inlets lie in rank 0's
    columns); an inlet across a seam adds the ranks' partial sums, which may round
    differently from the single-domain sum, so the [2, 1] split is held to the same
    steps and a relative tolerance of 1e-5."""
    q0, bed = flowing(NX, NY, seed=5, dtype=np.float32)
    ref = _make((NX, NY), ("wall", "wall"), "float32", q0, bed)
    _add_inlets(ref, (0, NX, 0, NY))
    ref_steps = ref.run(T_END)
    want = ref.q_interior.detach().cpu().numpy()
    torch.cuda.synchronize()
    world = dims[0] * dims[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_inlet_rank, args=(world, _free_port(), out, dims), nprocs=world,
                           start_method="spawn", join=True)
        out = dict(out)
    assert ref_steps > 20
    for r in range(world):
        o = out[r]
        x0, x1, y0, y1 = o["block"]
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps)
        if dims == [1, 2]:
            np.testing.assert_array_equal(o["q"], want[:, x0:x1, y0:y1])
        else:
            np.testing.assert_allclose(o["q"], want[:, x0:x1, y0:y1], rtol=1e-5, atol=1e-6)


CNX, CNY, CDX, C_T_END = 72, 90, 3.0, 900.0


def _compressed_inputs():
    from geoswe_b200.synthetic import MANNING_CLASSES, fractal_bed, voronoi_classes
    z = fractal_bed(CNX, CNY, CDX, seed=6).astype(np.float32)
    mask = z < np.percentile(z, 60)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    cls_pad = np.pad(voronoi_classes(CNX, CNY, n_seeds=16, seed=6), 2, mode="edge")
    return z, mask, cls_pad, MANNING_CLASSES


def _compressed_run(z, mask, cls_pad, table, block, **kw):
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    x0, x1, y0, y1 = block
    s = Solver2D(Mesh2D(nx=x1 - x0, ny=y1 - y0, dx=CDX, dy=CDX, ngh=2),
                 Config(bc_x="fall", bc_y="fall", friction="manning"),
                 np.zeros((3, x1 - x0, y1 - y0), np.float32), z[x0:x1, y0:y1].copy(), **kw)
    s.set_inside_mask(mask[x0:x1, y0:y1])
    s.set_manning_table(cls_pad[x0:x1 + 4, y0:y1 + 4].copy(), table)
    cs = CompressedSolver.from_dense(s)
    cs.set_rain(RainfallForcing(time_s=[0.0, 300.0, 1e9], rate_mm_h=[60.0, 25.0, 25.0]))
    steps = cs.run(t_end=C_T_END)
    return cs, steps


def _compressed_rank(rank, world, port, out, dims):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from geoswe_b200.partition import block_of
        z, mask, cls_pad, table = _compressed_inputs()
        block = block_of(CNX, CNY, dims, (rank // dims[1], rank % dims[1]))
        cs, steps = _compressed_run(z, mask, cls_pad, table, block, comm=dist.group.WORLD, dims=dims)
        out[rank] = dict(block=block, steps=steps, t=cs.t, depth=cs.depth(), n_active=cs.n_active,
                         sent=sum(cs.flat_halo.send_cells(s) for s in ("x-", "x+", "y-", "y+")),
                         exchanges=cs.flat_halo.exchanges, inner=cs.n_bricks_inner, nb=cs.n_bricks)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dims", [[2, 1], [1, 2]])
def test_split_compressed_run_equals_single_domain(dims):
    z, mask, cls_pad, table = _compressed_inputs()
    ref, ref_steps = _compressed_run(z, mask, cls_pad, table, (0, CNX, 0, CNY))
    want = ref.depth()
    torch.cuda.synchronize()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_compressed_rank, args=(2, _free_port(), out, dims), nprocs=2,
                           start_method="spawn", join=True)
        out = dict(out)
    assert ref_steps > 20 and want.max() > 0.01
    assert sum(out[r]["n_active"] for r in range(2)) == ref.n_active
    for r in range(2):
        o = out[r]
        x0, x1, y0, y1 = o["block"]
        assert o["sent"] > 0 and o["exchanges"] >= ref_steps
        assert 0 < o["inner"] < o["nb"]          # the step overlaps the seam exchange
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps, o["t"], ref.t)
        np.testing.assert_array_equal(o["depth"], want[x0:x1, y0:y1])


def _forced_compressed(z, mask, cls_pad, table, block, ckpt=None, max_steps=10 ** 9, resume=False, **kw):
    """The compressed rain run of `block` with a ring stage, infiltration, a sponge band and
    a discharge inlet, each given by global coordinates and restricted to the block (a
    rank lists what lies in its own block; the inlet is listed, possibly empty, on every
    rank)."""
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    x0, x1, y0, y1 = block
    s = Solver2D(Mesh2D(nx=x1 - x0, ny=y1 - y0, dx=CDX, dy=CDX, ngh=2),
                 Config(bc_x="fall", bc_y="fall", friction="manning"),
                 np.zeros((3, x1 - x0, y1 - y0), np.float32), z[x0:x1, y0:y1].copy(), **kw)
    s.set_inside_mask(mask[x0:x1, y0:y1])
    s.set_manning_table(cls_pad[x0:x1 + 4, y0:y1 + 4].copy(), table)
    cs = CompressedSolver.from_dense(s)
    cs.set_rain(RainfallForcing(time_s=[0.0, 300.0, 1e9], rate_mm_h=[60.0, 25.0, 25.0]))
    ij = cs.ij_active
    gi, gj = ij[:, 0] + x0, ij[:, 1] + y0                   # global padded indices
    own = (ij[:, 0] >= 2) & (ij[:, 0] < 2 + x1 - x0) & (ij[:, 1] >= 2) & (ij[:, 1] < 2 + y1 - y0)
    # ring stage on the ring cells of global rows < 30 (owned by this block)
    ring = np.nonzero((cs.is_active == 0) & own & (gi < 30))[0]
    bed = cs._b[cs._slot].cpu().numpy()[ring].astype(np.float32)
    t_c = np.array([0.0, 450.0, 900.0])
    cs.set_ring(dict(i=ij[ring, 0], j=ij[ring, 1], bed=bed, wg=np.ones((ring.size, 1), np.float32), NG=1,
                     n=int(ring.size), t_common=t_c, stage_all=np.array([[14.0, 16.0, 15.0]], np.float32)))
    cs.set_infil({"tab": np.array([1e-6, 2e-6, 5e-7, 0.0], np.float32)})
    keep = np.ones((cs.nxp, cs.nyp), np.float32)
    band = (np.arange(cs.nxp)[:, None] + x0 >= 40) & (np.arange(cs.nxp)[:, None] + x0 < 44)
    keep[np.broadcast_to(band, keep.shape)] = 0.995
    cs.set_sponge({"keep": keep, "amb": np.zeros_like(keep)})
    g, a = cs.ghost_boundary_pairs()
    pick = (ij[a, 0] == ij[g, 0]) & (ij[a, 1] == ij[g, 1] + 1) & (gi[g] >= 20) & (gi[g] < 28) & own[g]
    cs.add_inflow(g[pick], a[pick], (0.0, 1.0), CDX, [0.0, 400.0, 900.0], [0.0, 3.0, 0.5])
    steps = cs.run(t_end=C_T_END, window=8, max_steps=max_steps, checkpoint_every_s=200.0 if ckpt else 0.0,
                   ckpt_dir=ckpt, resume=resume)
    return cs, steps, int(pick.sum())


def _forced_rank(rank, world, port, out, dims, ckpt, m):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from geoswe_b200.partition import block_of
        z, mask, cls_pad, table = _compressed_inputs()
        block = block_of(CNX, CNY, dims, (rank // dims[1], rank % dims[1]))
        # a run stopped by a step cap (no clipped step) with checkpoints on the way, then
        # fresh solvers resuming from them
        cs, steps, n_inlet = _forced_compressed(z, mask, cls_pad, table, block, ckpt=ckpt, max_steps=m,
                                                comm=dist.group.WORLD, dims=dims)
        cs2, steps2, _ = _forced_compressed(z, mask, cls_pad, table, block, ckpt=ckpt, resume=True,
                                            comm=dist.group.WORLD, dims=dims)
        out[rank] = dict(block=block, steps=steps + steps2, t=cs2.t, nsteps=cs2.nsteps, depth=cs2.depth(),
                         n_inlet=n_inlet)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


def test_split_compressed_run_with_forcings_and_checkpoints(tmp_path):
    """A split compressed run with a ring stage, infiltration, a sponge band, a discharge
    inlet and checkpoints (per-rank state files, meta written by rank 0), stopped by a
    step cap half-way and resumed from its checkpoint by fresh solvers: equals the single-domain
    run bit for bit (the inlet lies in one rank's block; the other ranks list it empty)."""
    import json
    z, mask, cls_pad, table = _compressed_inputs()
    ref, ref_steps, n_inlet = _forced_compressed(z, mask, cls_pad, table, (0, CNX, 0, CNY))
    want = ref.depth()
    torch.cuda.synchronize()
    dims = [2, 1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_forced_rank, args=(2, _free_port(), out, dims, str(tmp_path), ref_steps // 2), nprocs=2,
                           start_method="spawn", join=True)
        out = dict(out)
    meta = json.load(open(tmp_path / "ckpt_meta.json"))
    assert ref_steps > 20 and n_inlet > 0
    assert meta["nranks"] == 2 and meta["steps"] == ref_steps
    assert (tmp_path / "ckpt_r00.npz").exists() and (tmp_path / "ckpt_r01.npz").exists()
    assert sum(out[r]["n_inlet"] for r in range(2)) == n_inlet
    for r in range(2):
        o = out[r]
        x0, x1, y0, y1 = o["block"]
        assert o["nsteps"] == ref_steps and o["t"] == ref.t, (r, o["nsteps"], ref_steps, o["t"], ref.t)
        np.testing.assert_array_equal(o["depth"], want[x0:x1, y0:y1])


def _seam_inlet_compressed(z, mask, cls_pad, table, block, **kw):
    """The compressed rain run of `block` with one discharge inlet along the top edge of
    the active set, global padded columns [30, 64): across the y seam of a [1, 2] split."""
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    x0, x1, y0, y1 = block
    s = Solver2D(Mesh2D(nx=x1 - x0, ny=y1 - y0, dx=CDX, dy=CDX, ngh=2),
                 Config(bc_x="fall", bc_y="fall", friction="manning"),
                 np.zeros((3, x1 - x0, y1 - y0), np.float32), z[x0:x1, y0:y1].copy(), **kw)
    s.set_inside_mask(mask[x0:x1, y0:y1])
    s.set_manning_table(cls_pad[x0:x1 + 4, y0:y1 + 4].copy(), table)
    cs = CompressedSolver.from_dense(s)
    cs.set_rain(RainfallForcing(time_s=[0.0, 300.0, 1e9], rate_mm_h=[60.0, 25.0, 25.0]))
    ij = cs.ij_active
    gi, gj = ij[:, 0] + x0, ij[:, 1] + y0
    own = (ij[:, 0] >= 2) & (ij[:, 0] < 2 + x1 - x0) & (ij[:, 1] >= 2) & (ij[:, 1] < 2 + y1 - y0)
    g, a = cs.ghost_boundary_pairs()
    pick = ((ij[a, 0] == ij[g, 0] + 1) & (ij[a, 1] == ij[g, 1]) & own[g] & (gi[g] < 20)
            & (gj[g] >= 30) & (gj[g] < 64))
    cs.add_inflow(g[pick], a[pick], (1.0, 0.0), CDX, [0.0, 300.0, 900.0], [0.0, 4.0, 1.0])
    steps = cs.run(t_end=C_T_END)
    return cs, steps, int(pick.sum())


def _seam_inlet_rank(rank, world, port, out, dims):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from geoswe_b200.partition import block_of
        z, mask, cls_pad, table = _compressed_inputs()
        block = block_of(CNX, CNY, dims, (rank // dims[1], rank % dims[1]))
        cs, steps, n = _seam_inlet_compressed(z, mask, cls_pad, table, block, comm=dist.group.WORLD, dims=dims)
        out[rank] = dict(block=block, steps=steps, t=cs.t, depth=cs.depth(), n=n)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


def test_split_compressed_inlet_across_the_seam():
    """A compressed inlet with cells on both ranks, starting dry: its dry seed (bed range,
    cells at the minimum, largest seed depth) is reduced over the ranks once, as the
    reference does, so the dry phase equals the single-domain run; once wet, each rank
    sums its cells' depths and one all-reduce adds the two partial sums in double, while
    the single-domain run sums all cells in float (as the reference's split and single
    runs do), so the inlet weights differ in the last bit and the difference grows over
    the run's ~7500 wet/dry steps: the run is held to the same steps, the same volume
    to 1e-4, and depths within 1 cm (RMSE 1 mm). An inlet inside one rank is bitwise
    (the test above)."""
    z, mask, cls_pad, table = _compressed_inputs()
    ref, ref_steps, n = _seam_inlet_compressed(z, mask, cls_pad, table, (0, CNX, 0, CNY))
    want = ref.depth()
    torch.cuda.synchronize()
    dims = [1, 2]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_seam_inlet_rank, args=(2, _free_port(), out, dims), nprocs=2,
                           start_method="spawn", join=True)
        out = dict(out)
    assert ref_steps > 20 and n > 0
    assert out[0]["n"] > 0 and out[1]["n"] > 0 and out[0]["n"] + out[1]["n"] == n
    for r in range(2):
        o = out[r]
        x0, x1, y0, y1 = o["block"]
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps)
        d = o["depth"].astype(np.float64) - want[x0:x1, y0:y1]
        assert np.abs(d).max() <= 1e-2 and np.sqrt(np.mean(d * d)) <= 1e-3, (r, np.abs(d).max())
    vol = sum(float(out[r]["depth"].astype(np.float64).sum()) for r in range(2))
    assert abs(vol - float(want.astype(np.float64).sum())) <= 1e-4 * float(want.astype(np.float64).sum())


def _plain_compressed(z, mask, cls_pad, table, block, **kw):
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    x0, x1, y0, y1 = block
    s = Solver2D(Mesh2D(nx=x1 - x0, ny=y1 - y0, dx=CDX, dy=CDX, ngh=2),
                 Config(bc_x="fall", bc_y="fall", friction="manning"),
                 np.zeros((3, x1 - x0, y1 - y0), np.float32), z[x0:x1, y0:y1].copy(), **kw)
    s.set_inside_mask(mask[x0:x1, y0:y1])
    s.set_manning_table(cls_pad[x0:x1 + 4, y0:y1 + 4].copy(), table)
    cs = CompressedSolver.from_dense(s)
    cs.set_rain(RainfallForcing(time_s=[0.0, 300.0, 1e9], rate_mm_h=[60.0, 25.0, 25.0]))
    return cs


def _split_cache_rank(rank, world, port, out, dims, cdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        from geoswe_b200.compressed import CompressedSolver
        from geoswe_b200.partition import block_of
        z, mask, cls_pad, table = _compressed_inputs()
        block = block_of(CNX, CNY, dims, (rank // dims[1], rank % dims[1]))
        cs = _plain_compressed(z, mask, cls_pad, table, block, comm=dist.group.WORLD, dims=dims)
        cs.run(t_end=300.0)
        cs.save_cache(cdir)
        dist.barrier()
        ld = CompressedSolver.from_cache(cdir, comm=dist.group.WORLD, dims=dims)
        steps = ld.run(t_end=C_T_END)
        out[rank] = dict(block=block, steps=steps, t=ld.t, depth=ld.depth(), inner=ld.n_bricks_inner,
                         nb=ld.n_bricks, n_active=ld.n_active)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


def test_split_cache_saves_per_rank_and_reloads(tmp_path):
    """A split compressed run saves one cache directory per rank (the reference's r##
    layout: own cells active, placement, seam faces) and fresh solvers load it on the
    same ranks and continue: equal bit for bit to the single-domain run saved and
    reloaded at the same time."""
    import json
    from geoswe_b200.compressed import CompressedSolver
    z, mask, cls_pad, table = _compressed_inputs()
    one = _plain_compressed(z, mask, cls_pad, table, (0, CNX, 0, CNY))
    one.run(t_end=300.0)
    one.save_cache(tmp_path / "one")
    ref = CompressedSolver.from_cache(tmp_path / "one")
    ref_steps = ref.run(t_end=C_T_END)
    want = ref.depth()
    torch.cuda.synchronize()
    dims = [2, 1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_split_cache_rank, args=(2, _free_port(), out, dims, str(tmp_path / "split")),
                           nprocs=2, start_method="spawn", join=True)
        out = dict(out)
    for r in range(2):
        meta = json.load(open(tmp_path / "split" / f"r{r:02d}" / "meta.json"))
        assert meta["mpi"] and meta["nranks"] == 2 and len(meta["halo_faces"]) == 1
        assert meta["placement"]["i0"] == out[r]["block"][0] and meta["nx_glob"] == CNX
        assert (tmp_path / "split" / f"r{r:02d}" / "halo_f0_sfi.npy").exists()
    assert ref_steps > 20 and sum(out[r]["n_active"] for r in range(2)) == ref.n_active
    for r in range(2):
        o = out[r]
        x0, x1, y0, y1 = o["block"]
        assert 0 < o["inner"] < o["nb"]
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps)
        np.testing.assert_array_equal(o["depth"], want[x0:x1, y0:y1])
