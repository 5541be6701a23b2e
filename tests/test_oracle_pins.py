"""Pin the oracles to the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py running the reference package here).

* oracle.numpy_ref restates the reference's NumPy CPU path: it must reproduce the
  fixtures exactly (same operations, same order, same library).
* the C oracle restates the reference's GPU kernel text; the reference states that
  its CPU and GPU residuals agree to < 1e-12 in fp64 (tests/test_srm_cpu_matches_gpu.py
  of the reference), which is the bar here; full runs must take the same number of
  steps and stay within the stated depth tolerance.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import numpy_ref

G = np.load(Path(__file__).resolve().parent / "golden" / "reference_dense.npz")


def _eq(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_numpy_ref_residual_is_reference(dt):
    q = G[f"rhs40_{dt}_qpad"]
    b = G[f"rhs40_{dt}_bpad"]
    r = numpy_ref.residual(q, b, 2.0, 2.0, 9.81, 1e-6)
    assert r.dtype == q.dtype
    assert _eq(r, G[f"rhs40_{dt}"])


def test_c_oracle_residual_fp64_within_reference_contract():
    q = G["rhs40_float64_qpad"]
    b = G["rhs40_float64_bpad"]
    r = oracle.dense_rhs(q, b, 2.0, 2.0, 9.81, 1e-6)
    ref = G["rhs40_float64"]
    I = (slice(None), slice(2, -2), slice(2, -2))
    d = np.abs(r[I] - ref[I]).max()
    assert d < 1e-12, d
    assert np.abs(ref[I]).max() > 1e-3


def test_c_oracle_residual_fp32_close():
    q = G["rhs40_float32_qpad"]
    b = G["rhs40_float32_bpad"]
    r = oracle.dense_rhs(q, b, 2.0, 2.0, 9.81, 1e-6)
    ref = G["rhs40_float32"]
    I = (slice(None), slice(2, -2), slice(2, -2))
    scale = np.abs(ref[I]).max()
    assert np.abs(r[I] - ref[I]).max() <= 2e-5 * scale


def _dam(dt):
    q0 = G["dam_q0"]
    n = q0.shape[1]
    qp = np.zeros((3, n + 4, n + 4), dt)
    qp[:, 2:-2, 2:-2] = q0
    bp = np.zeros((n + 4, n + 4), dt)
    return qp, bp


@pytest.mark.parametrize("dt", ["float32", "float64"])
def test_numpy_ref_dam_break_is_reference(dt):
    qp, bp = _dam(np.dtype(dt))
    s = numpy_ref.NumpySolver2D(qp, bp, 2, 1.0, 1.0, kinds=["wall"] * 4)
    s.run(t_end=1e9, max_steps=60)
    assert s.t == float(G[f"dam_{dt}_t"])
    assert _eq(s.q[:, 2:-2, 2:-2], G[f"dam_{dt}_q"][:, 2:-2, 2:-2])


@pytest.mark.parametrize("dt", ["float32", "float64"])
def test_c_oracle_dam_break_vs_reference(dt):
    npd = np.dtype(dt)
    qp, bp = _dam(npd)
    o = oracle.OracleSolver2D(qp, bp, 2, 1.0, 1.0, kinds=["wall"] * 4)
    n = o.run(t_end=1e9, max_steps=60)
    assert n == 60
    ref = G[f"dam_{dt}_q"][:, 2:-2, 2:-2]
    h = o.q[0, 2:-2, 2:-2]
    err = np.abs(h - ref[0])
    tol = 1e-4 if dt == "float32" else 1e-10
    assert err.max() < tol, err.max()
    assert abs(o.t - float(G[f"dam_{dt}_t"])) < (1e-4 if dt == "float32" else 1e-9)


def _rain_setup(dt):
    z = G["rain_z"]
    nmap = G["rain_n"]
    nx, ny = z.shape
    npd = np.dtype(dt)
    qp = np.zeros((3, nx + 4, ny + 4), npd)
    bp = np.pad(z.astype(npd), 2, mode="edge")
    return z, nmap, qp, bp


@pytest.mark.parametrize("dt", ["float32", "float64"])
def test_numpy_ref_rain_on_terrain_is_reference(dt):
    z, nmap, qp, bp = _rain_setup(dt)
    npd = np.dtype(dt)
    s = numpy_ref.NumpySolver2D(qp, bp, 2, 3.0, 3.0, kinds=["wall", "fall", "wall", "wall"],
                                friction="manning", n_interior=np.pad(nmap, 2, mode="edge").astype(npd)[2:-2, 2:-2],
                                rain_times=[0.0, 1e9], rain_mm_h=[50.0, 50.0])
    n = s.run(t_end=1800.0)
    assert n == int(G[f"rain_{dt}_steps"])
    assert s.t == float(G[f"rain_{dt}_t"])
    assert _eq(s.q[:, 2:-2, 2:-2], G[f"rain_{dt}_q"][:, 2:-2, 2:-2])


def test_c_oracle_rain_on_terrain_vs_reference():
    """The reference's CPU path and its CUDA kernel text are two different algorithms at
    thin-film wet/dry fronts (the NumPy HLLC zeroes the velocity of a dry face state and
    clamps SM into [SL, SR]; the kernel keeps the cell velocity and does not clamp). On
    this steep rained terrain they separate within a few steps, so the kernel algorithm
    (the C oracle) is pinned to the NumPy fixtures by bounds, and its own fp32/fp64 runs
    must agree step for step -- as the reference's fp32/fp64 NumPy runs do."""
    runs = {}
    for dt in ("float32", "float64"):
        z, nmap, qp, bp = _rain_setup(dt)
        npd = np.dtype(dt)
        npad = np.pad(nmap, 2, mode="edge")
        vals, inv = np.unique(npad, return_inverse=True)
        o = oracle.OracleSolver2D(qp, bp, 2, 3.0, 3.0, kinds=["wall", "fall", "wall", "wall"], friction="manning",
                                  ncls=inv.reshape(npad.shape).astype(np.uint8), ntab=vals,
                                  rain_times=[0.0, 1e9], rain_frames=np.array([50.0 / 3.6e6] * 2, npd),
                                  rain_rmax=[50.0 / 3.6e6] * 2)
        runs[dt] = (o.run(t_end=1800.0), o.q[0, 2:-2, 2:-2].astype(np.float64), o.t)
    n32, h32, t32 = runs["float32"]
    n64, h64, t64 = runs["float64"]
    assert n32 == n64 and t32 == t64 == 1800.0
    assert float(np.sqrt(np.mean((h32 - h64) ** 2))) < 1e-5
    ref_steps = int(G["rain_float32_steps"])
    assert ref_steps == int(G["rain_float64_steps"])
    assert abs(n32 - ref_steps) <= 0.01 * ref_steps          # measured: 15915 vs 15996
    ref = G["rain_float32_q"][0, 2:-2, 2:-2]
    assert float(np.sqrt(np.mean((h32 - ref) ** 2))) < 0.01   # measured: 8.5 mm


def test_numpy_ref_stage_inflow_is_reference():
    """The NumPy restatement of the stage boundary and the inflow ghosts."""
    z2 = G["stage_z"]
    q0 = G["stage_q0"]
    nx, ny = z2.shape
    qp = np.zeros((3, nx + 4, ny + 4), np.float32)
    qp[:, 2:-2, 2:-2] = q0
    bp = np.pad(z2.astype(np.float32), 2, mode="edge")
    cells = np.argwhere(np.eye(1, nx, 0, dtype=bool).T.repeat(ny, axis=1)) + 2
    o = oracle.OracleSolver2D(qp, bp, 2, 2.0, 2.0, kinds=["wall"] * 4, friction="manning", manning_n=0.03,
                              stages=[dict(cells=cells, time_s=[0.0, 600.0], stage_m=[1.0, 1.4],
                                           bed=z2[0, :])],
                              inflows=[dict(i=np.full(6, nx + 1), j=np.arange(12, 18) + 2, nx=-1.0, ny=0.0, ds=2.0,
                                            t=np.array([0.0, 100.0, 400.0]), q=np.array([0.0, 5.0, 1.0]))])
    n = o.run(t_end=200.0)
    assert n == int(G["stage_steps"])
    ref = G["stage_q"][0, 2:-2, 2:-2]
    assert float(np.sqrt(np.mean((o.q[0, 2:-2, 2:-2].astype(np.float64) - ref) ** 2))) <= 5e-4


def test_pow_m43_accuracy():
    xs = np.concatenate([np.geomspace(1e-6, 1e2, 2001), [1.0, 2.0, 0.5]]).astype(np.float32)
    ex = xs.astype(np.float64) ** (-4.0 / 3.0)
    got = np.array([oracle.pow_m43(x) for x in xs])
    ulp = np.spacing(ex.astype(np.float32)).astype(np.float64)
    assert (np.abs(got - ex) / ulp).max() <= 1.9
    got64 = np.array([oracle.pow_m43(float(x), np.float64) for x in xs])
    assert np.max(np.abs(got64 - ex) / ex) < 2e-15      # a few double ulp
