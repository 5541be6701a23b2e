"""Compressed (flat) mesh on the GPU: bit-exact against the flat C oracle (which walks
the reference's int16 neighbour table), and against the dense kernel."""
import numpy as np
import pytest

import oracle
from tests._cases import flowing, same

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dense(q0, bed, mask, dx=2.0, **cfgkw):
    from geoswe_b200 import Config, Mesh2D, Solver2D
    nx, ny = bed.shape
    kw = dict(bc_x="fall", bc_y="fall", arith="portable")   # the oracle's Manning power
    kw.update(cfgkw)
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=2), Config(**kw), q0, bed)
    if mask is not None:
        s.set_inside_mask(mask)
    return s


def _blob_mask(nx, ny, seed=3):
    from geoswe_b200.synthetic import dilate_cross
    rng = np.random.default_rng(seed)
    m = np.zeros((nx, ny), bool)
    m[rng.integers(4, nx - 4, 12), rng.integers(4, ny - 4, 12)] = True
    m = dilate_cross(m, 9)
    m[:3, :] = m[-3:, :] = False
    m[:, :3] = m[:, -3:] = False
    return m


@pytest.mark.parametrize("bh", [4, 16])
def test_flat_residual_bitwise_dense_and_oracle(bh):
    from geoswe_b200.compressed import CompressedSolver
    q0, bed = flowing(70, 97, seed=12, dtype=np.float32)
    mask = _blob_mask(70, 97)
    s = _dense(q0, bed, mask)
    s.run(t_end=1e9, max_steps=5)                      # a non-trivial fixed state
    s.apply_bc()
    r_dense = s.residual().cpu().numpy()
    cs = CompressedSolver.from_dense(s, brick_h=bh)
    r_flat = cs.residual().cpu().numpy()
    act = cs.is_active != 0
    ij = cs.ij_active
    for c in range(3):
        assert same(r_flat[c][act], r_dense[c][ij[act, 0], ij[act, 1]]), c
    assert np.abs(r_flat[0][act]).max() > 0
    q = [cs.flat(c).cpu().numpy() for c in range(3)]
    b = cs._b[cs._slot].cpu().numpy()
    r_or = oracle.flat_rhs(cs.nbr, cs.is_active, q, b, 2.0, 9.81, 1e-6)
    assert same(r_flat, r_or)


@pytest.mark.parametrize("linf", [False, True])
def test_flat_run_bitwise_oracle(linf):
    from geoswe_b200 import RainfallForcing
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import MANNING_CLASSES, fractal_bed, voronoi_classes
    nx, ny, dx = 72, 90, 3.0
    z = fractal_bed(nx, ny, dx, seed=6).astype(np.float32)
    mask = z < np.percentile(z, 60)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    cls = voronoi_classes(nx, ny, n_seeds=16, seed=6)
    s = _dense(np.zeros((3, nx, ny), np.float32), z, mask, dx=dx, friction="manning")
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES)
    cs = CompressedSolver.from_dense(s, cfl_linf=linf)
    rf = RainfallForcing(time_s=[0.0, 600.0, 1e9], rate_mm_h=[50.0, 20.0, 20.0])
    cs.set_rain(rf)
    q = [cs.flat(c).cpu().numpy() for c in range(3)]
    b = cs._b[cs._slot].cpu().numpy()
    ncls = cs._ncls[cs._slot].cpu().numpy()
    o = oracle.OracleFlat(cs.nbr, cs.is_active, q, b, dx, ncls=ncls, ntab=MANNING_CLASSES, linf=linf,
                          rain_times=rf.time_s, rain_table=(np.asarray(rf.rate_mm_h) / 3.6e6).astype(np.float32)[:, None],
                          rain_lookup=np.zeros(cs.n_stored, np.int64))
    if linf:
        n_g = cs.run(t_end=1500.0)
        n_o = o.run(t_end=1500.0)
        assert n_g == n_o and n_g > 10
    else:
        # interval by interval: a new t_end per call, calls starting on either buffer,
        # one captured window replayed throughout
        n_g = [cs.run(t_end=t) for t in (250.0, 700.0, 1100.0, 1500.0)]
        n_o = [o.run(t_end=t) for t in (250.0, 700.0, 1100.0, 1500.0)]
        assert n_g == n_o and sum(n_g) > 10 and any(k % 2 for k in n_g)
        assert len(cs._graph_cache) == 1
    assert cs.t == o.t
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), o.q[c]), c


def test_row_segments_change_no_bit():
    """Splitting each brick's rows among 2 or 4 warps (GswFlatArgs.segments) gives the
    same residual and the same run as one warp per brick."""
    from geoswe_b200 import RainfallForcing
    from geoswe_b200.compressed import CompressedSolver
    q0, bed = flowing(70, 97, seed=12, dtype=np.float32)
    mask = _blob_mask(70, 97)
    out = []
    for segs in (1, 2, 4):
        s = _dense(q0, bed, mask, friction="manning", manning_n=0.03)
        cs = CompressedSolver.from_dense(s)
        cs.set_rain(RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[30.0, 30.0]))
        cs.segments = segs
        r = cs.residual().cpu().numpy()
        n = cs.run(t_end=60.0)
        out.append((r, n, cs.t, [cs.flat(c).cpu().numpy() for c in range(3)]))
    for r, n, t, q in out[1:]:
        assert same(r, out[0][0])
        assert n == out[0][1] > 10 and t == out[0][2]
        for c in range(3):
            assert same(q[c], out[0][3][c]), c


def test_dense_masked_run_equals_flat_run():
    """With the dense solver's velocity norm (cfl_linf) and a mask away from the edges,
    the dense run over the whole grid and the compressed run take the same steps and
    end in the same state on the active cells (the reference's equivalence contract,
    tests/test_gpu_compressed_equiv.py, bit for bit here)."""
    from geoswe_b200.compressed import CompressedSolver
    n = 80
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    r = np.hypot(i - 40, j - 38)
    bed = (0.002 * r ** 2).astype(np.float32)           # a bowl
    h = np.where(r < 10, 1.5, 0.0) + np.maximum(0.8 - bed, 0.0)
    q0 = np.stack([h, 0 * h, 0 * h]).astype(np.float32)
    mask = r < 30
    sd = _dense(q0, bed, mask, dx=1.0, friction="manning", manning_n=0.03)
    cs = CompressedSolver.from_dense(_dense(q0, bed, mask, dx=1.0, friction="manning", manning_n=0.03),
                                     cfl_linf=True)
    nd = sd.run(t_end=40.0)
    nf = cs.run(t_end=40.0)
    assert nd == nf
    hd = sd.depth()
    hf = cs.depth()
    assert same(hf[mask], hd[mask])


def _inlet_pairs(cs, n_cells):
    """The first `n_cells` ghost/active pairs whose active neighbour lies at +i (inward
    normal (1, 0)) and whose ghost bed is not below the neighbour's (an inlet the water
    can leave), in canonical order."""
    g, a = cs.ghost_boundary_pairs()
    ij = cs.ij_active
    b = cs._b[cs._slot].cpu().numpy()
    d = ij[a] - ij[g]
    sel = np.nonzero((d[:, 0] == 1) & (d[:, 1] == 0) & (b[g] >= b[a]))[0][:n_cells]
    return g[sel], a[sel]


@pytest.mark.parametrize("n_cells", [1, 5])
def test_flat_inflow_run_bitwise_oracle(n_cells):
    """A discharge inlet on the compressed mesh (dry start: relief seed and critical
    depth, then the depth-weighted split) against the oracle's restatement of the flat
    loop's inlet block."""
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import fractal_bed
    nx, ny, dx = 64, 70, 3.0
    z = fractal_bed(nx, ny, dx, seed=9).astype(np.float32)
    mask = z < np.percentile(z, 70)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    s = _dense(np.zeros((3, nx, ny), np.float32), z, mask, dx=dx, friction="manning", manning_n=0.035)
    cs = CompressedSolver.from_dense(s)
    g, a = _inlet_pairs(cs, n_cells)
    assert g.size == n_cells
    t_k = [0.0, 300.0, 900.0, 1800.0]
    q_k = [0.0, 12.0, 20.0, 4.0]
    cs.add_inflow(g, a, (1.0, 0.0), dx, t_k, q_k)
    q = [cs.flat(c).cpu().numpy() for c in range(3)]
    b = cs._b[cs._slot].cpu().numpy()
    o = oracle.OracleFlat(cs.nbr, cs.is_active, q, b, dx, ntab=[np.float32(0.035)], dt_max=4.0)
    o.add_inflow(g, a, (1.0, 0.0), dx, t_k, q_k)
    n_g = cs.run(t_end=700.0, dt_max=4.0)           # a dry start has no wave speed to limit dt
    n_o = o.run(t_end=700.0)
    assert n_g == n_o and n_g > 20
    assert cs.t == o.t
    h = cs.flat(0).cpu().numpy()
    assert h[cs.is_active != 0].sum() > 0          # water entered
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), o.q[c]), c


def test_flat_ring_stage_tidal_bitwise_oracle():
    """Everywhere-wet sinusoidal bed with a tidal stage on the x- ghost ring (one gauge,
    weight 1): the compressed run against the oracle's restatement of ring_bc_flat."""
    import warnings
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import tidal_case
    nx, ny, dx = 60, 70, 25.0
    h, z = tidal_case(nx, ny, dx=dx, seed=4)
    q0 = np.stack([h, np.zeros_like(h), np.zeros_like(h)]).astype(np.float32)
    s = _dense(q0, z, None, dx=dx, bc_x="wall", bc_y="wall", friction="manning", manning_n=0.03)
    s.apply_bc()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        cs = CompressedSolver.from_dense(s, track_max_depth=False)
    ij = cs.ij_active
    ids = np.nonzero(ij[:, 0] < 2)[0]
    b = cs._b[cs._slot].cpu().numpy()
    t_c = np.arange(0.0, 4000.0, 300.0)
    stage = (1.5 + 0.3 * np.sin(2 * np.pi * t_c / 2400.0)).astype(np.float32)[None, :]
    ring = dict(i=ij[ids, 0], j=ij[ids, 1], bed=b[ids], wg=np.ones((ids.size, 1), np.float32), NG=1,
                n=int(ids.size), t_common=t_c, stage_all=stage)
    cs.set_ring(ring)
    q = [cs.flat(c).cpu().numpy() for c in range(3)]
    o = oracle.OracleFlat(cs.nbr, cs.is_active, q, b, dx, ntab=[np.float32(0.03)])
    o.set_ring(ids, b[ids], ring["wg"], t_c, stage)
    n_g = cs.run(t_end=900.0)
    n_o = o.run(t_end=900.0)
    assert n_g == n_o and n_g > 20
    assert cs.t == o.t
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), o.q[c]), c
    assert abs(float(cs.flat(1).cpu().numpy()[cs.is_active != 0].max())) > 0   # the tide drives a flow


def test_empty_mask_refused_like_the_reference():
    """An inside mask with no cell: the reference's CompressedSWE raises ValueError
    (no interior neighbors); so does from_dense."""
    from geoswe_b200.compressed import CompressedSolver
    q0, bed = flowing(30, 31, seed=2, dtype=np.float32)
    s = _dense(q0, bed, np.zeros((30, 31), bool))
    with pytest.raises(ValueError, match="no interior neighbors"):
        CompressedSolver.from_dense(s)


def test_library_slot_map_equals_the_solvers():
    """The host entry point gsw_bricks_slot_of gives the canonical-to-slot map the
    solver builds on the device."""
    from geoswe_b200 import _lib as L
    from geoswe_b200.compressed import CompressedSolver
    q0, bed = flowing(70, 97, seed=12, dtype=np.float32)
    cs = CompressedSolver.from_dense(_dense(q0, bed, _blob_mask(70, 97)))
    ij = np.ascontiguousarray(cs.ij_active, np.int32)
    bij = np.ascontiguousarray(cs._bij.cpu().numpy(), np.int32)
    slot = np.empty(len(ij), np.int64)
    lib = L.lib()
    assert lib.gsw_bricks_slot_of(ij.ctypes.data, len(ij), bij.ctypes.data, len(bij), cs.brick_h, cs.nxp, cs.nyp,
                                  slot.ctypes.data) == 0
    assert np.array_equal(slot, cs._slot.cpu().numpy())


@pytest.mark.parametrize("where", ["depth", "bed"])
def test_nonfinite_state_raises(where):
    """A NaN depth (caught by the initial wave speed) or a NaN bed (the step makes the
    NaN, the step's own wave-speed key carries it) stops the flat loop with
    FloatingPointError, as the reference's dt_from_lam does."""
    from geoswe_b200 import RainfallForcing
    from geoswe_b200.compressed import CompressedSolver
    q0, bed = flowing(40, 50, seed=4, dtype=np.float32)
    s = _dense(q0, bed, _blob_mask(40, 50), friction="manning", manning_n=0.03)
    cs = CompressedSolver.from_dense(s)
    cs.set_rain(RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[20.0, 20.0]))
    k = int(np.nonzero(cs.is_active)[0][len(np.nonzero(cs.is_active)[0]) // 2])
    slot = int(cs.slot_of[k])
    if where == "depth":
        cs._q[cs._cur][0][slot] = float("nan")
    else:
        cs._b[slot] = float("nan")
    with pytest.raises(FloatingPointError):
        cs.run(t_end=60.0)
