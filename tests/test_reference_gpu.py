"""The product's kernels against the reference's own GPU kernels, on the B200.

oracle/ref_build.py compiles the reference's assembled kernel text (captured from the
reference package) into oracle/_ref/libref_{fma,strict}.so; oracle/ref_runner.py drives
them with the reference's loop. "strict" is compiled without FMA contraction, like the
product, so the residual must agree bit for bit; "fma" is the reference as NVRTC builds
it by default, which may contract a*b+c, so values agree to rounding level and runs are
held to the stated step-count and depth bars.
"""
import numpy as np
import pytest

from oracle import ref_runner
from tests._cases import flowing, pad_state, rough_partly_dry, same

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_runner.available("fma"),
                                 reason="oracle/_ref not built (needs the reference tree at build time)")]

torch = pytest.importorskip("torch")


def _gsw_residual(q0, bed, dtype, ngh=2, dx=2.0):
    from geoswe_b200 import Config, Mesh2D, Solver2D
    nx, ny = bed.shape
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=ngh), Config(bc_x="wall", bc_y="wall", dtype=dtype), q0, bed)
    s.apply_bc()
    return s.residual().cpu().numpy(), s


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("case", ["ref40", "flow"])
def test_residual_bitwise_vs_reference_kernel_strict(dtype, case):
    npd = np.dtype(dtype)
    q0, bed = rough_partly_dry(40, 40, 7, npd) if case == "ref40" else flowing(70, 97, 11, npd)
    r_g, s = _gsw_residual(q0, bed, dtype)
    qpad = s.q.cpu().numpy().copy()
    r_ref = ref_runner.ref_residual(qpad, s.b.cpu().numpy().copy(), 2.0, 2.0, 9.81, 1e-6, variant="strict")
    I = (slice(None), slice(2, -2), slice(2, -2))
    assert same(r_g[I], r_ref[I])


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_residual_vs_reference_kernel_fma(dtype):
    npd = np.dtype(dtype)
    q0, bed = flowing(70, 97, 11, npd)
    r_g, s = _gsw_residual(q0, bed, dtype)
    r_ref = ref_runner.ref_residual(s.q.cpu().numpy().copy(), s.b.cpu().numpy().copy(), 2.0, 2.0, 9.81, 1e-6,
                                    variant="fma")
    I = (slice(None), slice(2, -2), slice(2, -2))
    scale = np.abs(r_ref[I]).max()
    tol = 5e-6 if dtype == "float32" else 1e-13
    assert np.abs(r_g[I] - r_ref[I]).max() <= tol * scale


@pytest.mark.parametrize("variant", ["strict", "fma"])
def test_dam_break_run_vs_reference_gpu(variant):
    """Circular dam break (walls, no friction, CFL 0.5): the same number of steps to the
    same time; strict compilation agrees bit for bit."""
    from geoswe_b200 import Config, Mesh2D, Solver2D
    from geoswe_b200.synthetic import dam_break
    n = 256
    q0, bed = dam_break(n, radius=32.0)
    s = Solver2D(Mesh2D(nx=n, ny=n, dx=1.0, dy=1.0, ngh=2), Config(bc_x="wall", bc_y="wall"), q0, bed)
    qp, bp = pad_state(q0.astype(np.float32), bed.astype(np.float32), 2, np.float32)
    r = ref_runner.RefDenseGPU(qp, bp, 2, 1.0, 1.0, kinds=["wall"] * 4, variant=variant)
    t_end = 30.0
    n_g = s.run(t_end=t_end)
    n_r = r.run(t_end=t_end)
    assert n_g == n_r
    assert s.t == r.t == t_end
    hg = s.q[0].cpu().numpy()[2:-2, 2:-2].astype(np.float64)
    hr = r.q[0].cpu().numpy()[2:-2, 2:-2].astype(np.float64)
    if variant == "strict":
        assert same(s.q.cpu().numpy()[:, 2:-2, 2:-2], r.q.cpu().numpy()[:, 2:-2, 2:-2])
    else:
        assert float(np.sqrt(np.mean((hg - hr) ** 2))) < 1e-5
        assert np.abs(hg - hr).max() < 1e-3


def test_rain_on_terrain_run_vs_reference_gpu():
    """Rain on fractal terrain with 4 Manning classes and one open edge: step count and
    state against the reference's own fused-step kernel, compiled strictly and with FMA
    contraction. The product (Manning's power by powf, as the reference text) equals
    the strict build bit for bit. Thin films on steep terrain amplify rounding, so the
    reference's two builds differ from each other: the product takes the FMA build's
    step count and stays within twice the reference's own build-to-build spread of it."""
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.synthetic import MANNING_CLASSES, fractal_bed, voronoi_classes
    nx, ny, dx = 96, 80, 3.0
    z = fractal_bed(nx, ny, dx, seed=5).astype(np.float32)
    cls = voronoi_classes(nx, ny, n_seeds=24, seed=5)
    cfg = Config(bc_x="wall", bc_y="wall", bc={"x+": "fall"}, friction="manning",
                 rainfall_forcing=RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[50.0, 50.0]))
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=2), cfg, np.zeros((3, nx, ny), np.float32), z)
    clsp = np.pad(cls, 2, mode="edge")
    s.set_manning_table(clsp, MANNING_CLASSES)
    qp, bp = pad_state(np.zeros((3, nx, ny), np.float32), z, 2, np.float32)
    t_end = 900.0
    n_g = s.run(t_end=t_end)
    hg = s.q[0].cpu().numpy()[2:-2, 2:-2].astype(np.float64)
    out = {}
    for variant in ("strict", "fma"):
        r = ref_runner.RefDenseGPU(qp, bp, 2, dx, dx, kinds=["wall", "fall", "wall", "wall"], ncls=clsp,
                                   ntab=MANNING_CLASSES, friction=True, rain_rate=50.0 / 3.6e6, variant=variant)
        n_r = r.run(t_end=t_end)
        out[variant] = (n_r, r.q[0].cpu().numpy()[2:-2, 2:-2].astype(np.float64), r.q.cpu().numpy()[:, 2:-2, 2:-2])
    rm = lambda a, b: float(np.sqrt(np.mean((a - b) ** 2)))
    spread = rm(out["strict"][1], out["fma"][1])
    print(f"\nsteps gsw={n_g} ref_strict={out['strict'][0]} ref_fma={out['fma'][0]}; RMSE gsw-strict="
          f"{rm(hg, out['strict'][1]):.3g} gsw-fma={rm(hg, out['fma'][1]):.3g} strict-fma={spread:.3g} m")
    assert n_g == out["strict"][0] == out["fma"][0]
    assert same(s.q.cpu().numpy()[:, 2:-2, 2:-2], out["strict"][2])
    assert rm(hg, out["fma"][1]) <= max(5e-4, 2.0 * spread)
