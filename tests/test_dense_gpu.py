"""Dense fused step on the GPU against the C oracle (bit-for-bit).

The oracle (oracle/gsw_oracle.c) evaluates the reference kernel text per cell with
four faces; the kernel shares each face between its two cells. Both use separately
rounded IEEE operations, so every comparison here is exact equality (-0 == +0). The
solvers run with arith="portable": the oracle restates Manning's h^(-4/3) as the
portable Newton iteration (a CPU cannot reproduce CUDA's powf); the default "exact"
arithmetic, powf included, is checked against the reference's own kernel in
test_reference_gpu.py.
"""

import numpy as np
import pytest

import oracle
from tests._cases import flowing, pad_state, rough_partly_dry, same

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _solver(q0, bed, dtype, ngh=2, dx=2.0, dy=2.0, **cfgkw):
    from geoswe_b200 import Config, Mesh2D, Solver2D
    nx, ny = bed.shape
    mesh = Mesh2D(nx=nx, ny=ny, dx=dx, dy=dy, ngh=ngh)
    kw = dict(bc_x="wall", bc_y="wall", dtype=dtype, h_min=1e-6, arith="portable")
    kw.update(cfgkw)
    cfg = Config(**kw)
    return Solver2D(mesh, cfg, q0, bed)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("case,ngh", [("ref40", 2), ("flow", 2), ("flow", 4)])
@pytest.mark.parametrize("masked", [False, True])
def test_residual_matches_oracle(dtype, case, ngh, masked):
    npd = np.dtype(dtype)
    if case == "ref40":
        q0, bed = rough_partly_dry(40, 40, seed=7, dtype=npd)
    else:
        q0, bed = flowing(70, 97, seed=11, dtype=npd)
    s = _solver(q0, bed, dtype, ngh=ngh)
    mask = None
    if masked:
        mask = np.random.default_rng(5).random(bed.shape) < 0.7
        s.set_inside_mask(mask)
    s.apply_bc()
    r_gpu = s.residual().cpu().numpy()
    qp, bp = pad_state(q0, bed, ngh, npd)
    oracle.bc_fill(qp, ngh, ["wall"] * 4)
    mp = None
    if masked:
        mp = np.zeros(qp.shape[1:], np.uint8)
        mp[ngh:-ngh, ngh:-ngh] = mask
    r_cpu = oracle.dense_rhs(qp, bp, 2.0, 2.0, 9.81, 1e-6, mask=mp)
    assert np.abs(r_cpu).max() > 0
    for k in range(3):
        assert same(r_gpu[k], r_cpu[k]), f"component {k}: max |diff| {np.abs(r_gpu[k] - r_cpu[k]).max()}"


STEP_VARIANTS = [
    dict(),
    dict(friction="table"),
    dict(friction="field"),
    dict(friction="scalar"),
    dict(friction="table", rain="uniform"),
    dict(friction="table", rain="gridded", mask=True),
    dict(rain="uniform", mask=True, keep_h=False),
    dict(friction="table", quad=False, vcap=0.5),
]


def _configure(s, q0, bed, var, ngh, npd):
    """Apply a step variant to the solver and return the oracle's matching kwargs."""
    from geoswe_b200 import RainfallForcing
    nx, ny = bed.shape
    rng = np.random.default_rng(21)
    kw = dict(kinds=["wall"] * 4, h_min=1e-6, vcap=var.get("vcap", 15.0), quad=var.get("quad", True),
              keep_h=var.get("keep_h", True))
    s.cfg.friction_velocity_cap_ms = var.get("vcap", 15.0)
    s.cfg.friction_quadratic_alpha = var.get("quad", True)
    s.cfg.wetdry_keep_h = var.get("keep_h", True)
    fr = var.get("friction")
    if fr == "table":
        cls = rng.integers(0, 4, size=bed.shape).astype(np.uint8)
        clsp = np.pad(cls, ngh, mode="edge")
        tab = np.array([0.025, 0.04, 0.06, 0.1])
        s.cfg.friction = "manning_implicit"
        s.set_manning_table(clsp, tab)
        kw.update(friction="manning", ncls=clsp, ntab=tab)
    elif fr == "field":
        nf = (0.02 + 0.08 * rng.random(bed.shape))
        nfp = np.pad(nf, ngh, mode="edge").astype(npd)
        s.set_manning(nf)
        kw.update(friction="manning", nfield=nfp)
    elif fr == "scalar":
        s.cfg.friction = "manning_implicit"
        s.cfg.manning_n = 0.035
        s._invalidate()
        kw.update(friction="manning", manning_n=0.035)
    if var.get("mask"):
        m = rng.random(bed.shape) < 0.8
        s.set_inside_mask(m)
        mp = np.zeros((nx + 2 * ngh, ny + 2 * ngh), np.uint8)
        mp[ngh:-ngh, ngh:-ngh] = m
        kw.update(mask=mp)
    rain = var.get("rain")
    if rain == "uniform":
        rf = RainfallForcing(time_s=[0.0, 50.0, 1e9], rate_mm_h=[80.0, 30.0, 0.0])
        s.cfg.rainfall_forcing = rf
        s._invalidate()
        fr_ = rf.frames(npd)
        kw.update(rain_times=rf.time_s, rain_frames=fr_, rain_gridded=False,
                  rain_rmax=[float(r) / 3.6e6 for r in rf.rate_mm_h])
    elif rain == "gridded":
        rate = rng.random((3, nx, ny)) * 100.0
        rf = RainfallForcing(time_s=[0.0, 40.0, 90.0], rate_mm_h=rate)
        s.cfg.rainfall_forcing = rf
        s._invalidate()
        fr_ = rf.frames(npd)
        kw.update(rain_times=rf.time_s, rain_frames=fr_, rain_gridded=True,
                  rain_rmax=[float(f.max()) for f in fr_])
    return kw


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("vi", range(len(STEP_VARIANTS)))
def test_step_matches_oracle(dtype, vi):
    var = STEP_VARIANTS[vi]
    npd = np.dtype(dtype)
    ngh = 2
    q0, bed = flowing(64, 75, seed=vi + 1, dtype=npd)
    s = _solver(q0, bed, dtype, ngh=ngh)
    kw = _configure(s, q0, bed, var, ngh, npd)
    qp, bp = pad_state(q0, bed, ngh, npd)
    o = oracle.OracleSolver2D(qp, bp, ngh, 2.0, 2.0, **kw)
    for k in range(4):
        dt_o = o.cfl_dt()
        dt_g = s.cfl_dt()
        assert dt_o == dt_g, (k, dt_o, dt_g)
        s.step(dt_g)
        o.step(dt_o)
        g = s.q.cpu().numpy()
        n = ngh
        for c in range(3):
            assert same(g[c][n:-n, n:-n], o.q[c][n:-n, n:-n]), f"step {k} comp {c} var {var}"
    assert same(s.max_depth(), o.max_h[n:-n, n:-n])


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_run_dam_break_matches_oracle(dtype):
    """Config-1 shape (walls, no friction, CFL 0.5, h_min 1e-6) at 96^2 for 150 steps,
    through the device-resident loop and CUDA graphs."""
    from geoswe_b200.synthetic import dam_break
    npd = np.dtype(dtype)
    q0, bed = dam_break(96, radius=12.0)
    s = _solver(q0, bed, dtype, ngh=2, dx=1.0, dy=1.0)
    qp, bp = pad_state(q0.astype(npd), bed.astype(npd), 2, npd)
    o = oracle.OracleSolver2D(qp, bp, 2, 1.0, 1.0, kinds=["wall"] * 4, h_min=1e-6)
    n_g = s.run(t_end=1.0e6, max_steps=150)
    n_o = o.run(t_end=1.0e6, max_steps=150)
    assert n_g == n_o == 150
    assert s.t == o.t
    g = s.q.cpu().numpy()
    for c in range(3):
        assert same(g[c][2:-2, 2:-2], o.q[c][2:-2, 2:-2])


def test_run_rain_friction_open_edge_matches_oracle():
    """Rain-on-terrain shape: fractal bed, 4-class Manning, dry start, uniform rain,
    x+ open ('fall'), other faces walls; runs to a fixed t_end (rain step limit and
    the final clip exercised)."""
    from geoswe_b200 import RainfallForcing
    from geoswe_b200.synthetic import fractal_bed, voronoi_classes
    nx, ny, dx = 80, 100, 3.0
    z = fractal_bed(nx, ny, dx, seed=4)
    cls = voronoi_classes(nx, ny, n_seeds=16, seed=4)
    q0 = np.zeros((3, nx, ny))
    s = _solver(q0, z, "float32", ngh=2, dx=dx, dy=dx, bc={"x+": "fall"})
    s.set_manning(np.array([0.025, 0.04, 0.06, 0.1])[cls])
    rf = RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0])
    s.cfg.rainfall_forcing = rf
    s._invalidate()
    qp, bp = pad_state(q0.astype(np.float32), z.astype(np.float32), 2, np.float32)
    clsp = np.pad(np.array([0.025, 0.04, 0.06, 0.1])[cls], 2, mode="edge")
    vals, inv = np.unique(clsp, return_inverse=True)
    o = oracle.OracleSolver2D(qp, bp, 2, dx, dx, kinds=["wall", "fall", "wall", "wall"], h_min=1e-6,
                              friction="manning", ncls=inv.reshape(clsp.shape).astype(np.uint8), ntab=vals,
                              rain_times=rf.time_s, rain_frames=rf.frames(np.float32),
                              rain_rmax=[50.0 / 3.6e6] * 2)
    t_end = 3000.0
    n_g = s.run(t_end=t_end)
    n_o = o.run(t_end=t_end)
    assert n_g == n_o and n_g > 20
    assert s.t == o.t == t_end
    g = s.q.cpu().numpy()
    for c in range(3):
        assert same(g[c][2:-2, 2:-2], o.q[c][2:-2, 2:-2])


def test_graph_replay_equals_eager():
    from geoswe_b200 import Config, Mesh2D, Solver2D
    q0, bed = flowing(60, 61, seed=9, dtype=np.float32)
    out = []
    for graphs in (True, False):
        mesh = Mesh2D(nx=60, ny=61, dx=2.0, dy=2.0, ngh=2)
        s = Solver2D(mesh, Config(bc_x="wall", bc_y="extrapolate"), q0, bed, use_graphs=graphs)
        s.run(t_end=1e9, max_steps=37, window=8)
        out.append((s.t, s.nsteps, s.q.cpu().numpy().copy()))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1] == 37
    assert same(out[0][2][:, 2:-2, 2:-2], out[1][2][:, 2:-2, 2:-2])


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_host_loop_equals_device_loop(dtype):
    """run(callback=...) -- cfl_dt read back and step(dt) from the host each step, the
    reference's own loop (solver.py:2975-3027) -- equals the device loop bit for bit,
    with rain (its dt limit) and friction on."""
    from geoswe_b200 import Config, Mesh2D, Solver2D
    q0, bed = flowing(52, 47, seed=4, dtype=np.dtype(dtype))
    out = []
    for host in (True, False):
        mesh = Mesh2D(nx=52, ny=47, dx=2.0, dy=2.5, ngh=2)
        s = Solver2D(mesh, Config(bc_x="wall", bc_y="fall", dtype=dtype, friction="manning",
                                  manning_n=0.03, rainfall=80.0 / 3.6e6), q0, bed)
        calls = []
        n = s.run(t_end=9.0, callback=(lambda solver, k: calls.append(k)) if host else None)
        out.append((n, s.t, s.q_interior.cpu().numpy().copy()))
        if host:
            assert calls == list(range(1, n + 1))
    assert out[0][0] == out[1][0] > 20 and out[0][1] == out[1][1] == 9.0
    assert same(out[0][2], out[1][2])


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_windows_tile_the_step(dtype):
    """The step launched as an interior window plus four bands (what a split run does
    around its halo exchange) writes the same state and wave speed as one launch."""
    import ctypes as C
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _ptr, _stream
    q0, bed = flowing(58, 45, seed=8, dtype=np.dtype(dtype))
    s = _solver(q0, bed, dtype, friction="manning", manning_n=0.03, rainfall=70.0 / 3.6e6)
    s.run(t_end=1e9, max_steps=9)
    T = s._tables()
    s._write_state()
    p = s._dt_params(t_end=float("inf"), fixed_dt=0.05)
    L.call("gsw_dt_finalize", C.byref(p), _ptr(s._state), _stream())
    src = s._buf[s._cur]
    L.call("gsw_bc_fill", C.byref(s._bc_args(src)), _stream())
    g, nxp, nyp = 2, s.nxp, s.nyp
    outs, lams = [], []
    for windows in ([(0, 0, 0, 0)],
                    [(g + 2, nxp - g - 2, g + 2, nyp - g - 2), (g, g + 2, g, nyp - g), (nxp - g - 2, nxp - g, g, nyp - g),
                     (g + 2, nxp - g - 2, g, g + 2), (g + 2, nxp - g - 2, nyp - g - 2, nyp - g)]):
        out = torch.zeros_like(src)
        s._lam_view.zero_()
        a = s._dense_args(src, out, T)
        a.max_h = None
        for w in windows:
            a.row_lo, a.row_hi, a.col_lo, a.col_hi = w
            L.call("gsw_dense_step", C.byref(a), _stream())
        outs.append(out[:, g:nxp - g, g:nyp - g].cpu().numpy())
        lams.append(int(s._lam_view.item()))
    assert same(outs[0], outs[1]) and lams[0] == lams[1] != 0
    assert np.abs(outs[0][0]).max() > 0.1


def test_segmented_runs_reuse_one_graph():
    """run() called interval by interval (new t_end each call, odd step counts, so the
    calls start on either buffer) equals one run to the last t_end bit for bit, and
    replays one captured window throughout: the dt rule is read from device memory and
    a run starting on buffer 1 takes one step before the window."""
    from geoswe_b200 import Config, Mesh2D, Solver2D
    q0, bed = flowing(60, 61, seed=9, dtype=np.float32)
    runs = []
    for ends in ([7.0, 13.5, 21.0, 30.0], [30.0]):
        mesh = Mesh2D(nx=60, ny=61, dx=2.0, dy=2.0, ngh=2)
        s = Solver2D(mesh, Config(bc_x="wall", bc_y="extrapolate"), q0, bed)
        n = [s.run(t_end=t, window=8) for t in ends]
        assert len(s._graph_cache) == 1
        runs.append((s.t, sum(n), s.q.cpu().numpy().copy(), n))
    assert any(k % 2 for k in runs[0][3])
    assert runs[0][0] == runs[1][0] == 30.0
    # the clipped steps at each interval end differ from the single run's, so compare
    # against a run over the same intervals without graphs instead of the single run
    mesh = Mesh2D(nx=60, ny=61, dx=2.0, dy=2.0, ngh=2)
    e = Solver2D(mesh, Config(bc_x="wall", bc_y="extrapolate"), q0, bed, use_graphs=False)
    ne = [e.run(t_end=t, window=8) for t in [7.0, 13.5, 21.0, 30.0]]
    assert ne == runs[0][3] and e.t == runs[0][0]
    assert same(e.q.cpu().numpy()[:, 2:-2, 2:-2], runs[0][2][:, 2:-2, 2:-2])


def test_nonfinite_state_raises():
    q0, bed = flowing(40, 40, seed=2, dtype=np.float32)
    s = _solver(q0, bed, "float32")
    s.q[0, 20, 20] = float("nan")          # a NaN depth reaches the wave speed
    with pytest.raises(FloatingPointError):
        s.run(t_end=1e9, max_steps=10)


@pytest.mark.parametrize("kinds", [("extrapolate",) * 4, ("wall", "fall", "periodic", "periodic"),
                                   ("periodic", "periodic", "wall", "extrapolate")])
def test_boundary_kinds_match_oracle(kinds):
    from geoswe_b200 import Config, Mesh2D, Solver2D
    ngh = 3
    q0, bed = flowing(50, 66, seed=13, dtype=np.float32)
    bc = dict(zip(("x-", "x+", "y-", "y+"), kinds))
    bx = "periodic" if kinds[0] == "periodic" else "wall"
    by = "periodic" if kinds[2] == "periodic" else "wall"
    mesh = Mesh2D(nx=50, ny=66, dx=2.0, dy=2.0, ngh=ngh)
    s = Solver2D(mesh, Config(bc_x=bx, bc_y=by, bc=bc), q0, bed)
    qp = np.zeros((3, 50 + 2 * ngh, 66 + 2 * ngh), np.float32)
    qp[:, ngh:-ngh, ngh:-ngh] = q0
    bp = s.b.cpu().numpy().copy()
    o = oracle.OracleSolver2D(qp, bp, ngh, 2.0, 2.0, kinds=list(kinds), h_min=1e-6)
    s.run(t_end=1e9, max_steps=25)
    o.run(t_end=1e9, max_steps=25)
    g = s.q.cpu().numpy()
    for c in range(3):
        assert same(g[c][ngh:-ngh, ngh:-ngh], o.q[c][ngh:-ngh, ngh:-ngh])


def test_stage_boundary_and_inflow_match_oracle():
    from geoswe_b200 import Config, Mesh2D, Solver2D, StageBoundary
    from geoswe_b200.synthetic import fractal_bed
    nx, ny, ngh, dx = 64, 48, 2, 2.0
    z = fractal_bed(nx, ny, dx, seed=8, zmax=2.0).astype(np.float32)
    q0 = np.zeros((3, nx, ny), np.float32)
    q0[0] = np.maximum(1.0 - z, 0.0)
    mesh = Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=ngh)
    edge = np.zeros((nx, ny), bool)
    edge[0, :] = True
    sb = StageBoundary.from_mask(edge, mesh, z, time_s=[0.0, 600.0], stage_m=[1.0, 1.4])
    cfg = Config(bc_x="wall", bc_y="wall", stage_boundary=sb, friction="manning", manning_n=0.03, arith="portable")
    s = Solver2D(mesh, cfg, q0, z)
    ii = np.full(6, nx - 1 + ngh)
    jj = np.arange(20, 26) + ngh
    s.add_inflow(ii, jj, (-1.0, 0.0), dx, [0.0, 100.0, 400.0], [0.0, 5.0, 1.0])
    qp, bp = pad_state(q0, z, ngh, np.float32)
    o = oracle.OracleSolver2D(qp, bp, ngh, dx, dx, kinds=["wall"] * 4, h_min=1e-6, friction="manning",
                              manning_n=0.03,
                              stages=[dict(cells=sb.cells, time_s=sb.time_s, stage_m=sb.stage_m, bed=sb.bed_b)],
                              inflows=[dict(i=ii, j=jj, nx=-1.0, ny=0.0, ds=dx, t=np.array([0.0, 100.0, 400.0]),
                                            q=np.array([0.0, 5.0, 1.0]))])
    n_g = s.run(t_end=300.0)
    n_o = o.run(t_end=300.0)
    assert n_g == n_o
    g = s.q.cpu().numpy()
    for c in range(3):
        assert same(g[c][ngh:-ngh, ngh:-ngh], o.q[c][ngh:-ngh, ngh:-ngh]), c
