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
        refused = False
        try:
            s.add_inflow([2], [3], (1.0, 0.0), 2.0, [0.0, 1.0], [1.0, 1.0])
        except NotImplementedError:
            refused = True
        if host_loop:
            steps = s.run(T_END, callback=lambda solver, k: None)
        else:
            steps = s.run(T_END)
        q = s.q_interior.detach().cpu().numpy().copy()
        out[rank] = dict(block=(x0, x1, y0, y1), steps=steps, t=s.t, q=q, refused=refused,
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
        assert o["refused"], "add_inflow on a split run must raise"
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps, o["t"], ref.t)
        assert o["exchanges"] >= ref_steps and o["launches"] > 0
        np.testing.assert_array_equal(o["q"], want[:, x0:x1, y0:y1])


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
                         exchanges=cs.flat_halo.exchanges)
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
        assert o["steps"] == ref_steps and o["t"] == ref.t, (r, o["steps"], ref_steps, o["t"], ref.t)
        np.testing.assert_array_equal(o["depth"], want[x0:x1, y0:y1])
