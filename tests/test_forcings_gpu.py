"""The flat loop's per-step forcings on the GPU: landcover infiltration, the sponge band,
Green-Ampt infiltration with the linear-reservoir drain (fused, Green-Ampt only, drain
only), the stage clamp and the karst drain cap. Each is applied once to a wet state and
compared bit for bit with the reference's own kernel text compiled with strict IEEE
rounding (oracle/_ref), the drain's __expf included, and close to the same
text compiled with FMA contraction as NVRTC compiles it; a run with all of them (Green-Ampt-only mode) is compared
bit for bit with the oracle's restatement of the flat loop."""
import numpy as np
import pytest

import oracle
from oracle import ref_runner
from tests._cases import same

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_runner.available("fma"), reason="oracle/_ref not built")]
torch = pytest.importorskip("torch")


def _solver(seed=5, nx=52, ny=60, dx=4.0):
    import warnings
    from geoswe_b200 import Config, Mesh2D, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import fractal_bed, voronoi_classes, MANNING_CLASSES
    z = (0.3 * fractal_bed(nx, ny, dx, seed=seed)).astype(np.float32)
    mask = z < np.quantile(z, 0.75)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    rng = np.random.default_rng(seed)
    h = np.where(mask, np.maximum(np.quantile(z, 0.5) - z, 0.0) + 0.02 * rng.random(z.shape), 0.0)
    q0 = np.stack([h, 0.05 * (rng.random(z.shape) - 0.5) * (h > 0), 0.05 * (rng.random(z.shape) - 0.5) * (h > 0)])
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=dx, dy=dx, ngh=2), Config(bc_x="fall", bc_y="fall", friction="manning", arith="portable"),
                 q0.astype(np.float32), z)
    s.set_inside_mask(mask)
    cls = voronoi_classes(nx, ny, n_seeds=10, seed=seed)
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return CompressedSolver.from_dense(s), rng


def _forcing_inputs(cs, rng):
    N, nxp, nyp = cs.N_stored, cs.nxp, cs.nyp
    pad_cls = rng.integers(0, 3, (nxp, nyp)).astype(np.uint8)
    F_pad = (rng.random((nxp, nyp)) * 0.02).astype(np.float32)
    Fmax_pad = (0.01 + rng.random((nxp, nyp)) * 0.05).astype(np.float32)
    tau_pad = np.where(rng.random((nxp, nyp)) < 0.5, 1.0 / 3600.0, 0.0).astype(np.float32)
    ga = dict(cls_pad=pad_cls, Ks_t=np.array([1e-6, 5e-6, 0.0], np.float32),
              psi_t=np.array([0.09, 0.2, 0.1], np.float32), dth_t=np.array([0.3, 0.25, 0.2], np.float32),
              F_pad=F_pad, Fmax_pad=Fmax_pad, inv_tau_pad=tau_pad)
    keep = np.ones((nxp, nyp), np.float32)
    amb = np.zeros((nxp, nyp), np.float32)
    keep[:8, :] = np.linspace(0.8, 1.0, 8, dtype=np.float32)[:, None]
    amb[:8, :] = (1 - keep[:8, :]) * np.float32(0.4)
    ij = cs.ij_active
    act = np.nonzero(cs.is_active != 0)[0]
    pick = rng.choice(act, 40, replace=False)
    hc = (cs.flat(0).cpu().numpy()[pick] * 0.5).astype(np.float32)
    return ga, dict(keep=keep, amb=amb), dict(rows=ij[pick[:20], 0], cols=ij[pick[:20], 1], hmax=hc[:20]), \
        dict(idx=pick[20:], h_tgt_arr=hc[20:]), np.array([2e-6, 0.0, 4e-6, 1e-6], np.float32)


def _canon(cs, t):
    return t[cs._slot]


@pytest.mark.parametrize("mode", ["fused", "ga", "drain"])
def test_each_forcing_once_matches_reference_kernel(mode):
    import ctypes as C
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _ptr, _stream
    cs, rng = _solver()
    ga, sp, cl, dr, infil = _forcing_inputs(cs, rng)
    ga["mode"] = mode
    cs.set_infil(dict(tab=infil)).set_sponge(sp).set_ga_drain(ga).set_clamp(cl).set_drain(dr)
    dt = 7.5
    st = L.GswLoopState()
    st.dt, st.dt_f32 = dt, float(np.float32(dt))
    cs._state.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))), dtype=torch.uint8))
    q = cs._q[cs._cur]
    sl = cs._slot
    act = torch.from_numpy(cs.is_active.copy()).cuda()
    ncls = cs._ncls[sl].contiguous()
    f = cs._forcing
    canon_of = cs._canonical_of_slot()
    g = f["ga"]
    Fmax = g["Fmax"][sl].contiguous()
    tau = g["inv_tau"][sl].contiguous()
    gcls = g["cls"][sl].contiguous()
    which = {"fused": "ga_drain", "ga": "ga", "drain": "drain_tau"}[mode]

    def reference(variant):
        """The reference kernels, in the reference loop's order, on canonical arrays."""
        rq = [x[sl].clone() for x in q]
        F_ref = g["F"][sl].clone()
        kw = dict(variant=variant)
        ref_runner.ref_forcing("infiltrate", rq, cls=ncls, t0=f["infil"], act=act, dt=dt, h_min=cs.h_min, **kw)
        ref_runner.ref_forcing("sponge", rq, idx=canon_of[f["sponge"]["slots"]].to(torch.int32),
                               a0=f["sponge"]["keep"], a1=f["sponge"]["amb"], **kw)
        ref_runner.ref_forcing(which, rq, cls=gcls, t0=g["Ks"], t1=g["psi"], t2=g["dth"], F=F_ref, Fmax=Fmax,
                               inv_tau=tau, act=act, dt=dt, **kw)
        ref_runner.ref_forcing("clamp", rq, idx=canon_of[f["clamp"]["slots"]].to(torch.int32),
                               a0=f["clamp"]["hmax"], **kw)
        ref_runner.ref_forcing("drain_cap", rq, idx=canon_of[f["drain"]["slots"]].to(torch.int32),
                               a0=f["drain"]["htgt"], **kw)
        return rq, F_ref

    # strict IEEE build: bit for bit; nvcc-default build (FMA contraction, as the
    # reference runs under NVRTC): close (the Green-Ampt quadratic rounds differently)
    rq, F_ref = reference("strict")
    rq_fma, F_fma = reference("fma")
    # the product, in place on the brick storage
    for phase in (0, 1):
        L.call("gsw_flat_forcings", C.byref(cs._forcing_args(q, phase)), _stream())
    torch.cuda.synchronize()
    for c in range(3):
        assert same(q[c][sl].cpu().numpy(), rq[c].cpu().numpy()), c
        np.testing.assert_allclose(q[c][sl].cpu().numpy(), rq_fma[c].cpu().numpy(), rtol=1e-5, atol=1e-8)
    assert same(g["F"][sl].cpu().numpy(), F_ref.cpu().numpy())
    np.testing.assert_allclose(g["F"][sl].cpu().numpy(), F_fma.cpu().numpy(), rtol=1e-5, atol=1e-8)


def test_run_with_forcings_matches_oracle():
    cs, rng = _solver(seed=8)
    ga, sp, cl, dr, infil = _forcing_inputs(cs, rng)
    ga["mode"] = "ga"
    cs.set_infil(dict(tab=infil)).set_sponge(sp).set_ga_drain(ga).set_clamp(cl).set_drain(dr)
    sl = cs._slot
    canon_of = cs._canonical_of_slot()
    f = cs._forcing
    q = [cs.flat(c).cpu().numpy() for c in range(3)]
    o = oracle.OracleFlat(cs.nbr, cs.is_active, q, cs._b[sl].cpu().numpy(), cs.dx,
                          ncls=cs._ncls[sl].cpu().numpy(), ntab=cs._ntab.cpu().numpy())
    npy = lambda t: t.cpu().numpy()
    o.set_forcings(infil_tab=infil,
                   sponge=(npy(canon_of[f["sponge"]["slots"]]), npy(f["sponge"]["keep"]), npy(f["sponge"]["amb"])),
                   ga=dict(mode="ga", cls=npy(f["ga"]["cls"][sl]), Ks=npy(f["ga"]["Ks"]), psi=npy(f["ga"]["psi"]),
                           dth=npy(f["ga"]["dth"]), F=npy(f["ga"]["F"][sl]).copy(), Fmax=npy(f["ga"]["Fmax"][sl]),
                           inv_tau=None),
                   clamp=(npy(canon_of[f["clamp"]["slots"]]), npy(f["clamp"]["hmax"])),
                   drain=(npy(canon_of[f["drain"]["slots"]]), npy(f["drain"]["htgt"])))
    n_g = cs.run(t_end=600.0)
    n_o = o.run(t_end=600.0)
    assert n_g == n_o and n_g > 20
    assert cs.t == o.t
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), o.q[c]), c
    assert same(f["ga"]["F"][sl].cpu().numpy(), o.forcings["ga"]["F"])
