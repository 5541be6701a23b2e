"""Generate the golden fixtures of tests/golden/ by running the reference itself.

    python tests/golden/make_golden.py [--ref <reference checkout>/src]

(default: oracle.ref_build.reference_src(), i.e. $GEOSWE_REFERENCE_SRC or the build
host's checkout)

Imports the reference package (geoswe) with its NumPy backend from the read-only
reference tree and records, for small seeded inputs, what its own CPU path computes:
residuals (fp64 and fp32), short runs of its time loop (final state, time, dt
sequence) with walls / open edge / rain / Manning / stage / inflow, and, through a
NumPy stand-in for CuPy, its compressed-mesh tables. The outputs are committed as
.npz; the tests compare the oracle (and through it the GPU kernels) against them.
Nothing at test time reads the reference tree.
"""
from __future__ import annotations

import argparse
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(src):
    os.environ["GEOSWE_BACKEND"] = "numpy"
    sys.path.insert(0, str(src))
    import geoswe  # noqa: F401
    return geoswe


def _rough(nx, ny, seed=7):
    rng = np.random.default_rng(seed)
    bed = rng.random((nx, ny)) * 1.2
    q0 = np.zeros((3, nx, ny))
    q0[0] = np.maximum(0.8 - bed, 0.0)
    wet = q0[0] > 1e-6
    q0[1] = (rng.random((nx, ny)) - 0.5) * 0.04 * wet
    q0[2] = (rng.random((nx, ny)) - 0.5) * 0.04 * wet
    return q0, bed


def residual_cases(G, out):
    from geoswe import Config, Mesh2D, Solver2D
    q0, bed = _rough(40, 40, 7)
    for dt in ("float64", "float32"):
        mesh = Mesh2D(nx=40, ny=40, dx=2.0, dy=2.0, ngh=2)
        cfg = Config(pde="baseline", flux="hllc", recon="first", well_balanced=True, wb_method="srm",
                     time="euler", cfl=0.5, bc_x="wall", bc_y="wall", dtype=dt, h_min=1e-6)
        s = Solver2D(mesh, cfg, q0, bed)
        s._apply_bc()
        rhs = np.asarray(s._rhs(s.q))
        out[f"rhs40_{dt}"] = rhs
        out[f"rhs40_{dt}_qpad"] = np.asarray(s.q)
        out[f"rhs40_{dt}_bpad"] = np.asarray(s.b)
    out["rhs40_q0"] = q0
    out["rhs40_bed"] = bed


def _fractal(nx, ny, dx, seed):
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.fftfreq(ny)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    amp = np.zeros_like(k)
    amp[k > 0] = k[k > 0] ** -1.5
    z = np.real(np.fft.ifft2((rng.standard_normal((nx, ny)) + 1j * rng.standard_normal((nx, ny))) * amp))
    z = (z - z.min()) / (z.max() - z.min()) * 40.0
    return z + 0.002 * ((np.arange(nx) + 0.5) * dx)[:, None]


def run_cases(G, out):
    from geoswe import Config, Mesh2D, RainfallForcing, Solver2D, StageBoundary
    from geoswe.bc import apply_bc_2d, apply_bc_2d_face

    # dam break (walls, no friction) -- the small-scale shape of the 512^2 case
    n = 64
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    r = np.hypot(i - (n - 1) / 2.0, j - (n - 1) / 2.0)
    q0 = np.zeros((3, n, n))
    q0[0] = np.where(r < 8.0, 2.0, 0.5)
    bed = np.zeros((n, n))
    for dt in ("float32", "float64"):
        mesh = Mesh2D(nx=n, ny=n, dx=1.0, dy=1.0, ngh=2)
        cfg = Config(bc_x="wall", bc_y="wall", cfl=0.5, h_min=1e-6, dtype=dt)
        s = Solver2D(mesh, cfg, q0, bed)
        dts = []
        s.run(t_end=1e9, max_steps=60, callback=lambda so, k: dts.append(so.last_dt if hasattr(so, "last_dt") else None))
        out[f"dam_{dt}_q"] = np.asarray(s.q)
        out[f"dam_{dt}_t"] = np.float64(s.t)
    out["dam_q0"] = q0

    # rain on terrain: fractal bed, 4-class Manning, dry start, x+ open, walls elsewhere
    nx, ny, dx = 48, 40, 3.0
    z = _fractal(nx, ny, dx, 4)
    rng = np.random.default_rng(4)
    cls = rng.integers(0, 4, size=(nx, ny))
    nmap = np.array([0.025, 0.04, 0.06, 0.1])[cls]

    class OpenEdge(Solver2D):
        def _apply_bc(self):
            apply_bc_2d(self.q, self.mesh.ngh, kind_x="wall", kind_y="wall")
            apply_bc_2d_face(self.q, self.mesh.ngh, "x+", "fall")
            self._fill_inflow_ghosts()

    for dt in ("float32", "float64"):
        mesh = Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=2)
        rf = RainfallForcing(time_s=np.array([0.0, 1e9]), rate_mm_h=np.array([50.0, 50.0]))
        cfg = Config(bc_x="wall", bc_y="wall", cfl=0.5, h_min=1e-6, dtype=dt, friction="manning",
                     rainfall_forcing=rf)
        s = OpenEdge(mesh, cfg, np.zeros((3, nx, ny)), z)
        s.set_manning(nmap)
        nsteps = s.run(t_end=1800.0)
        out[f"rain_{dt}_q"] = np.asarray(s.q)
        out[f"rain_{dt}_t"] = np.float64(s.t)
        out[f"rain_{dt}_steps"] = np.int64(nsteps)
        out[f"rain_{dt}_maxh"] = np.asarray(s.max_depth())
    out["rain_z"] = z
    out["rain_n"] = nmap

    # stage boundary on one edge + a discharge inlet on the opposite edge, fp32
    nx, ny, dx = 40, 32, 2.0
    z2 = _fractal(nx, ny, dx, 8) * (2.0 / 40.0)
    q0 = np.zeros((3, nx, ny))
    q0[0] = np.maximum(1.0 - z2, 0.0)
    mesh = Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=2)
    edge = np.zeros((nx, ny), bool)
    edge[0, :] = True
    sb = StageBoundary.from_mask(edge, mesh, z2, time_s=np.array([0.0, 600.0]), stage_m=np.array([1.0, 1.4]))
    cfg = Config(bc_x="wall", bc_y="wall", cfl=0.5, h_min=1e-6, dtype="float32", friction="manning",
                 manning_n=0.03, stage_boundary=sb)
    s = Solver2D(mesh, cfg, q0, z2)
    ii = np.full(6, nx - 1 + 2)
    jj = np.arange(12, 18) + 2
    s.add_inflow(ii, jj, (-1.0, 0.0), dx, np.array([0.0, 100.0, 400.0]), np.array([0.0, 5.0, 1.0]))
    nsteps = s.run(t_end=200.0)
    out["stage_q"] = np.asarray(s.q)
    out["stage_t"] = np.float64(s.t)
    out["stage_steps"] = np.int64(nsteps)
    out["stage_z"] = z2
    out["stage_q0"] = q0


def _cupy_standin():
    """A NumPy-backed stand-in for the `cupy` module, enough for the compressed-mesh
    builders to run on the CPU."""
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            try:
                setattr(cp, name, getattr(np, name))
            except Exception:
                pass
    cp.ndarray = np.ndarray
    cp.asnumpy = lambda a: np.asarray(a)
    cp.get_default_memory_pool = lambda: types.SimpleNamespace(free_all_blocks=lambda: None)
    cuda = types.ModuleType("cupy.cuda")
    cuda.runtime = types.SimpleNamespace(memGetInfo=lambda: (0, 0))
    cp.cuda = cuda
    sys.modules["cupy"] = cp
    sys.modules["cupy.cuda"] = cuda
    return cp


def mesh_cases(G, out):
    _cupy_standin()
    import geoswe.backend as B
    B.raw_kernel = lambda *a, **k: None
    from geoswe.mesh import Mesh2D
    from geoswe.compressed_rhs import CompressedSWE
    rng = np.random.default_rng(11)
    cases = {
        "blob": (rng.random((40, 30)) < 0.55),
        "band": np.zeros((48, 52), bool),
        "rect": np.zeros((30, 40), bool),
    }
    cases["band"][10:38, 5:47] = True
    cases["band"][20:30, 15:25] = False
    cases["rect"][4:26, 3:37] = True
    cases["single"] = np.zeros((7, 9), bool)          # one inside cell
    cases["single"][3, 4] = True
    cases["empty"] = np.zeros((6, 5), bool)           # no inside cell
    cases["edge"] = np.zeros((12, 10), bool)          # inside cells on the array edge: ring not covered
    for name, inside_int in cases.items():
        nxp, nyp = inside_int.shape[0] + 4, inside_int.shape[1] + 4
        inside = np.zeros((nxp, nyp), bool)
        inside[2:-2, 2:-2] = inside_int
        if name == "edge":
            inside[0:5, 3:8] = True
        mesh_pad = Mesh2D(nx=nxp, ny=nyp, dx=1.0, dy=1.0, ngh=0)
        out[f"mesh_{name}_inside"] = inside
        try:
            cs = CompressedSWE(mesh_pad, inside, ring=2)
        except ValueError as e:                       # the reference refuses this active set
            out[f"mesh_{name}_raises"] = np.str_(str(e))
            continue
        out[f"mesh_{name}_ij"] = np.asarray(cs.cm.ij_active)
        out[f"mesh_{name}_aid"] = np.asarray(cs.cm.active_id_padded)
        out[f"mesh_{name}_nbr32"] = np.asarray(cs.cm.neighbors)
        out[f"mesh_{name}_nbr16"] = np.asarray(cs.nbr)
        out[f"mesh_{name}_active"] = np.asarray(cs.is_active)
        out[f"mesh_{name}_covered"] = np.bool_(cs.fully_covered)


def cache_cases(G, out_dir):
    """A flat-mesh cache written by the reference's own save_cache (compressed_solver.py:
    2504-2560) for a small mesh with a wet state, a two-column rain table with a per-cell
    lookup and a two-gauge ring stage."""
    _cupy_standin()
    import geoswe.backend as B
    B.raw_kernel = lambda *a, **k: None
    B.elementwise_kernel = lambda *a, **k: None     # module-level kernels, never launched here
    from geoswe.mesh import Mesh2D
    from geoswe.compressed_rhs import CompressedSWE
    import geoswe.compressed_solver as CSol
    rng = np.random.default_rng(23)
    nx, ny, ngh, dx = 44, 50, 2, 5.0
    z = _fractal(nx, ny, dx, 23)[:, :] * 0.25
    inside_int = z < np.quantile(z, 0.7)
    inside_int[:3, :] = inside_int[-3:, :] = False
    inside_int[:, :3] = inside_int[:, -3:] = False
    nxp, nyp = nx + 2 * ngh, ny + 2 * ngh
    inside = np.zeros((nxp, nyp), bool)
    inside[ngh:-ngh, ngh:-ngh] = inside_int
    bp = np.pad(z, ngh, mode="edge").astype(np.float32)
    cs = CompressedSWE(Mesh2D(nx=nxp, ny=nyp, dx=1.0, dy=1.0, ngh=0), inside, ring=2)
    ij = np.asarray(cs.cm.ij_active)
    N = ij.shape[0]
    bed_f = bp[ij[:, 0], ij[:, 1]].astype(np.float32)
    eta = np.float32(np.quantile(z, 0.45))
    q0 = np.maximum(eta - bed_f, 0.0).astype(np.float32)
    q0 += (rng.random(N) * 0.02 * (q0 > 0)).astype(np.float32)
    q1 = ((rng.random(N) - 0.5) * 0.05 * (q0 > 0)).astype(np.float32)
    q2 = ((rng.random(N) - 0.5) * 0.05 * (q0 > 0)).astype(np.float32)
    act = np.asarray(cs.is_active)
    mcls = rng.integers(0, 3, N).astype(np.uint8)
    m_tab = np.array([0.03, 0.05, 0.08], np.float32)
    rain = dict(native_rate_dev=(np.array([[20.0, 60.0], [5.0, 40.0], [0.0, 10.0]]) / 3.6e6).astype(np.float32),
                lookup_flat=((ij[:, 1] // 10) % 2).astype(np.int32), t_s=np.array([0.0, 120.0, 400.0]))
    ring_ids = np.nonzero((act == 0) & (ij[:, 0] < nxp // 2))[0]
    w = rng.random((ring_ids.size, 2)).astype(np.float32)
    w /= w.sum(axis=1, keepdims=True)
    t_c = np.arange(0.0, 1200.0, 100.0)
    stage = np.stack([eta + 0.2 * np.sin(2 * np.pi * t_c / 600.0),
                      eta + 0.1 * np.cos(2 * np.pi * t_c / 900.0)]).astype(np.float32)
    ring = dict(rflat=ring_ids.astype(np.int32), rbed=bed_f[ring_ids], rwg=w.reshape(-1), t_common=t_c,
                stage_all=stage, NG=2, n=int(ring_ids.size))
    os.makedirs(out_dir, exist_ok=True)
    CSol.save_cache(str(out_dir), nbr=np.asarray(cs.nbr), is_active=act, ij_active=ij, nxp=nxp, nyp=nyp, ngh=ngh,
                    dx=dx, x0=0.0, y0=0.0, crs_wkt="", nx_glob=nx, ny_glob=ny, q0=q0, q1=q1, q2=q2, bed_f=bed_f,
                    sig_f=np.zeros(N, np.float32), mcls_f=mcls, m_tab=m_tab, inv_sig_f=np.ones(N, np.float32),
                    ring=ring, sponge=None, rain=rain, no_sigma=True, say=lambda *a, **k: None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    a = ap.parse_args()
    G = _import_reference(a.ref or _default_ref())
    out = {}
    residual_cases(G, out)
    run_cases(G, out)
    np.savez_compressed(HERE / "reference_dense.npz", **out)
    mesh_out = {}
    mesh_cases(G, mesh_out)
    np.savez_compressed(HERE / "reference_mesh.npz", **mesh_out)
    cache_cases(G, HERE / "reference_cache")
    for f in ("reference_dense.npz", "reference_mesh.npz"):
        print(f, (HERE / f).stat().st_size, "bytes")


def _default_ref():
    sys.path.insert(0, str(HERE.parents[1]))
    from oracle.ref_build import reference_src
    return str(reference_src())


def main_mesh(ref=None):
    """Only the mesh tables (reference_mesh.npz)."""
    G = _import_reference(ref or _default_ref())
    mesh_out = {}
    mesh_cases(G, mesh_out)
    np.savez_compressed(HERE / "reference_mesh.npz", **mesh_out)


if __name__ == "__main__":
    if "--mesh-only" in sys.argv:
        sys.argv.remove("--mesh-only")
        main_mesh()
    else:
        main()
