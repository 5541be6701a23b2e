"""Batched ensemble on the GPU: every member's trajectory equals its stand-alone
CompressedSolver run bit for bit (same steps, same state), with members of different
sizes, active sets, rain, Manning tables and end times advanced by one persistent
kernel per step."""
import numpy as np
import pytest

from tests._cases import same

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _member(seed, nx, ny, frac, peak, scale):
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import MANNING_CLASSES, fractal_bed, voronoi_classes
    z = fractal_bed(nx, ny, 3.0, seed=seed).astype(np.float32)
    mask = z < np.percentile(z, 100 * frac)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    cls = voronoi_classes(nx, ny, n_seeds=12, seed=seed)
    s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=3.0, dy=3.0, ngh=2),
                 Config(bc_x="fall", bc_y="fall", friction="manning"), np.zeros((3, nx, ny), np.float32), z)
    s.set_inside_mask(mask)
    s.set_manning_table(np.pad(cls, 2, mode="edge"), MANNING_CLASSES * scale)
    cs = CompressedSolver.from_dense(s)
    t = np.arange(0.0, 1800.0, 60.0)
    rate = peak * np.clip(1.0 - np.abs(t + 30.0 - 600.0) / 600.0, 0.0, None)
    cs.set_rain(RainfallForcing(time_s=t, rate_mm_h=rate))
    return cs


SPECS = [(1, 40, 50, 0.5, 80.0, 1.0), (2, 64, 64, 0.8, 40.0, 0.8), (3, 90, 70, 0.35, 120.0, 1.2),
         (4, 33, 120, 0.6, 60.0, 1.1)]


@pytest.mark.parametrize("segments", [1, 4])
def test_members_equal_standalone_runs(segments):
    """Members end at different times (the running-member list is rebuilt as each one
    finishes); row segments per brick change no bit."""
    from geoswe_b200.ensemble import Ensemble
    t_ends = [900.0, 600.0, 1200.0, 750.0]
    alone = [_member(*sp) for sp in SPECS]
    steps_alone = [cs.run(t_end=te) for cs, te in zip(alone, t_ends)]
    ens = Ensemble([_member(*sp) for sp in SPECS])
    ens.segments = segments
    steps = ens.run(t_end=t_ends, window=16)
    assert steps == steps_alone
    for k, cs in enumerate(alone):
        assert ens.members[k].t == cs.t
        for c in range(3):
            assert same(ens.flat(k, c).cpu().numpy(), cs.flat(c).cpu().numpy()), (k, c)


def test_second_run_continues():
    from geoswe_b200.ensemble import Ensemble
    alone = [_member(*sp) for sp in SPECS[:2]]
    for cs in alone:
        cs.run(t_end=300.0)
        cs.run(t_end=500.0)
    ens = Ensemble([_member(*sp) for sp in SPECS[:2]])
    ens.run(t_end=300.0, window=8)
    ens.run(t_end=500.0, window=8)
    for k, cs in enumerate(alone):
        assert ens.members[k].t == cs.t
        assert same(ens.flat(k, 0).cpu().numpy(), cs.flat(0).cpu().numpy())


def test_lean_step_equals_general_step_and_guards_its_premise():
    """Members in the production configuration take the compiled-in (lean) step; it
    equals the general step bit for bit. A member outside that configuration in a step
    forced lean is stopped with an error the host raises, not advanced wrongly."""
    from geoswe_b200.ensemble import Ensemble
    lean = Ensemble([_member(*sp) for sp in SPECS[:2]])
    general = Ensemble([_member(*sp) for sp in SPECS[:2]])
    assert lean.lean
    general.lean = False
    assert lean.run(t_end=400.0, window=8) == general.run(t_end=400.0, window=8)
    for k in range(2):
        for c in range(3):
            assert same(lean.flat(k, c).cpu().numpy(), general.flat(k, c).cpu().numpy()), (k, c)
    odd = _member(*SPECS[1])
    odd.cfl_linf = True
    mixed = Ensemble([_member(*SPECS[0]), odd])
    assert not mixed.lean
    mixed.lean = True
    with pytest.raises(RuntimeError, match="member 1 was stopped"):
        mixed.run(t_end=100.0, window=8)
