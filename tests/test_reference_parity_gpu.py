"""Parity with the reference's own GPU kernels at the benchmark configurations.

oracle/ref_build.py compiles the reference's kernel text, captured from its package,
without FMA contraction ("strict", the product's rounding) and with NVRTC's default
contraction ("fma", the reference as it runs). oracle/ref_runner.py drives them with
the reference's dense loop (RefDenseGPU) and its flat loop (RefFlatGPU). The product's
default arithmetic evaluates Manning's h^(-4/3) with CUDA's powf as the reference text
does, so every run here must equal the strict build bit for bit and take the fma
build's step count; against the fma build the depth RMSE is stated and held to the
0.05 cm bar.

Cases: the dam break of the small configuration at its full size (512 x 512, r = 64,
walls, no friction, 500 steps); a 512 x 512 crop of the rain-on-terrain 8192 x 8192
field (the same seeded bed and Manning classes the benchmark generates, x+ open,
50 mm/h) for 2000 steps, dense and on the compressed mesh (active set z below the
crop's 60th percentile, dilated 8 cells; both wave-speed norms); and the dense and
compressed residuals at a wet state of a 2048 x 2048 crop, identical to each other and
to the reference's residual kernel.
"""
import numpy as np
import pytest

from oracle import ref_runner
from tests._cases import pad_state, same

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_runner.available("strict"),
                                 reason="oracle/_ref not built (needs the reference tree at build time)")]
torch = pytest.importorskip("torch")

RMSE_BAR = 5e-4        # 0.05 cm, the depth tolerance against the reference


def _rmse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)))


@pytest.fixture(scope="module")
def field8192():
    """The rain-on-terrain bed of the 8192 x 8192 configuration (seed 0, float32)."""
    from geoswe_b200.synthetic import fractal_bed
    return fractal_bed(8192, 8192, 3.0, seed=0).astype(np.float32)


def _crop(field, n, i0=3000, j0=2000):
    from geoswe_b200.synthetic import voronoi_classes_window
    z = np.ascontiguousarray(field[i0:i0 + n, j0:j0 + n])
    cls = voronoi_classes_window(8192, 8192, i0, i0 + n, j0, j0 + n, seed=0)
    return z, cls


def _rain_solver(z, cls, **cfgkw):
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.synthetic import MANNING_CLASSES
    n = z.shape[0]
    cfg = Config(bc_x="wall", bc_y="wall", bc={"x+": "fall"}, friction="manning", cfl=0.5,
                 rainfall_forcing=RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0]), **cfgkw)
    s = Solver2D(Mesh2D(nx=n, ny=z.shape[1], dx=3.0, dy=3.0, ngh=2), cfg, np.zeros((3,) + z.shape, np.float32), z)
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES)
    return s


def test_config1_dam_break_full_size():
    """512 x 512 dam break, r = 64 cells, walls, no friction, CFL 0.5, 500 steps."""
    from geoswe_b200 import Config, Mesh2D, Solver2D
    from geoswe_b200.synthetic import dam_break
    n = 512
    q0, bed = dam_break(n, radius=64.0)
    s = Solver2D(Mesh2D(nx=n, ny=n, dx=1.0, dy=1.0, ngh=2), Config(bc_x="wall", bc_y="wall", cfl=0.5), q0, bed)
    n_g = s.run(t_end=1e9, max_steps=500)
    qp, bp = pad_state(q0.astype(np.float32), bed.astype(np.float32), 2, np.float32)
    out = {}
    for variant in ("strict", "fma"):
        r = ref_runner.RefDenseGPU(qp, bp, 2, 1.0, 1.0, kinds=["wall"] * 4, variant=variant)
        n_r = r.run(t_end=1e9, max_steps=500)
        out[variant] = (n_r, r.t, r.q.cpu().numpy()[:, 2:-2, 2:-2])
    g = s.q.cpu().numpy()[:, 2:-2, 2:-2]
    assert n_g == out["strict"][0] == out["fma"][0] == 500
    assert s.t == out["strict"][1]
    assert same(g, out["strict"][2])
    e = _rmse(g[0], out["fma"][2][0])
    print(f"\nconfig 1: depth RMSE vs the reference's fma build {e:.3g} m, max {np.abs(g[0] - out['fma'][2][0]).max():.3g} m")
    assert e <= RMSE_BAR


def test_config2_crop_dense_2000_steps(field8192):
    """Rain on terrain (4 Manning classes, x+ open, 50 mm/h, dry start), 2000 steps of a
    512 x 512 crop: bitwise against the strict build, Manning included."""
    from geoswe_b200.synthetic import MANNING_CLASSES
    z, cls = _crop(field8192, 512)
    s = _rain_solver(z, cls)
    n_g = s.run(t_end=1e9, max_steps=2000)
    qp, bp = pad_state(np.zeros((3,) + z.shape, np.float32), z, 2, np.float32)
    out = {}
    for variant in ("strict", "fma"):
        r = ref_runner.RefDenseGPU(qp, bp, 2, 3.0, 3.0, kinds=["wall", "fall", "wall", "wall"],
                                   ncls=np.pad(cls, 2, mode="edge"), ntab=MANNING_CLASSES, friction=True,
                                   rain_rate=50.0 / 3.6e6, variant=variant)
        n_r = r.run(t_end=1e9, max_steps=2000)
        out[variant] = (n_r, r.t, r.q.cpu().numpy()[:, 2:-2, 2:-2])
    g = s.q.cpu().numpy()[:, 2:-2, 2:-2]
    assert n_g == out["strict"][0] == out["fma"][0] == 2000
    assert s.t == out["strict"][1]
    assert same(g, out["strict"][2])
    e = _rmse(g[0], out["fma"][2][0])
    print(f"\nconfig 2 crop, dense: t = {s.t:.1f} s, depth RMSE vs the fma build {e:.3g} m, "
          f"max {np.abs(g[0] - out['fma'][2][0]).max():.3g} m")
    assert e <= RMSE_BAR


@pytest.mark.parametrize("linf", [False, True])
def test_config2_crop_compressed_2000_steps(field8192, linf):
    """The same crop on the compressed mesh (active set z < 60th percentile of the crop,
    dilated 8 cells), 2000 steps of the flat loop, against the reference's flat fused
    step + CFL kernel and its flat loop: bitwise against the strict build at every stored
    cell, same steps and time."""
    from geoswe_b200 import RainfallForcing
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import dilate_cross
    z, cls = _crop(field8192, 512)
    mask = dilate_cross(z < np.percentile(z, 60), 8)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    s = _rain_solver(z, cls)
    s.set_inside_mask(mask)
    cs = CompressedSolver.from_dense(s, cfl_linf=linf)
    rf = RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0])
    cs.set_rain(rf)
    q = [cs.flat(c).cpu().numpy() for c in range(3)]
    bed = cs._b[cs._slot].cpu().numpy()
    ncls = cs._ncls[cs._slot].cpu().numpy()
    table = (np.asarray(rf.rate_mm_h, np.float64) / 3.6e6).astype(np.float32)[:, None]
    n_g = cs.run(t_end=1e9, max_steps=2000)
    out = {}
    for variant in ("strict", "fma"):
        r = ref_runner.RefFlatGPU(cs.nbr, cs.is_active, q, bed, 3.0, n_cls=ncls, n_tab=cs._ntab.cpu().numpy(),
                                  linf=linf, rain_times=np.asarray(rf.time_s, np.float64), rain_table=table,
                                  rain_lookup=np.zeros(cs.n_stored, np.int32), variant=variant)
        n_r = r.run(t_end=1e9, max_steps=2000)
        out[variant] = (n_r, r.t, [r.q[c].cpu().numpy() for c in range(3)])
    g = [cs.flat(c).cpu().numpy() for c in range(3)]
    assert n_g == out["strict"][0] == out["fma"][0] == 2000
    assert cs.t == out["strict"][1]
    for c in range(3):
        assert same(g[c], out["strict"][2][c]), c
    act = cs.is_active != 0
    e = _rmse(g[0][act], out["fma"][2][0][act])
    print(f"\nconfig 2 crop, compressed (linf={linf}): {int(act.sum())} active cells, t = {cs.t:.1f} s, "
          f"depth RMSE vs the fma build {e:.3g} m")
    assert e <= RMSE_BAR


def test_config2_residuals_dense_compressed_reference_2048(field8192):
    """At a wet state of a 2048 x 2048 crop (water level at the crop's 40th bed percentile
    with seeded velocities, so wet/dry fronts everywhere), the dense residual, the
    compressed residual at active cells and the reference's residual kernel (strict) are
    identical."""
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import dilate_cross
    z, cls = _crop(field8192, 2048, i0=1024, j0=4096)
    rng = np.random.default_rng(11)
    h = np.maximum(np.percentile(z, 40) - z, 0.0).astype(np.float32)
    u = (rng.standard_normal(z.shape) * 0.5).astype(np.float32)
    v = (rng.standard_normal(z.shape) * 0.5).astype(np.float32)
    q0 = np.stack([h, h * u, h * v]).astype(np.float32)
    mask = dilate_cross(z < np.percentile(z, 60), 8)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    from geoswe_b200 import Config, Mesh2D, Solver2D
    s = Solver2D(Mesh2D(nx=2048, ny=2048, dx=3.0, dy=3.0, ngh=2),
                 Config(bc_x="wall", bc_y="wall", bc={"x+": "fall"}), q0, z)
    s.set_inside_mask(mask)
    s.apply_bc()
    r_dense = s.residual().cpu().numpy()
    cs = CompressedSolver.from_dense(s)
    r_flat = cs.residual().cpu().numpy()
    act = cs.is_active != 0
    ij = cs.ij_active
    nz = 0
    for c in range(3):
        d = r_dense[c][ij[act, 0], ij[act, 1]]
        assert same(r_flat[c][act], d), c
        nz = max(nz, int(np.count_nonzero(d)))
    assert nz > 0.3 * int(act.sum())
    m = np.zeros(s.q.shape[1:], np.uint8)
    m[2:-2, 2:-2] = mask
    r_ref = ref_runner.ref_residual(s.q.cpu().numpy().copy(), s.b.cpu().numpy().copy(), 3.0, 3.0, 9.81, 1e-6,
                                    variant="strict", mask=m)
    I = (slice(None), slice(2, -2), slice(2, -2))
    assert same(r_dense[I], r_ref[I])
