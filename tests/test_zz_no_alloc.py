"""gsw_ensemble_step_static (the ensemble step with its ticket counter in the library's
static device array) against gsw_ensemble_step with caller scratch: two calls in a row
from the same state give the same states and fields bit for bit, and the caller's
scratch argument is neither needed nor touched; and a whole loop (wave speed, dt rule,
static step) runs with no caller scratch at all, as a host without a device allocator
runs it. Collected last on purpose: the static variant's first call on a device does
its one-time setup here, after whatever the other test files ran."""
import ctypes as C

import numpy as np
import pytest

from tests._cases import same

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _ensemble():
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.ensemble import Ensemble
    from geoswe_b200.synthetic import MANNING_CLASSES, fractal_bed, voronoi_classes
    members = []
    for seed, nx, ny in ((3, 48, 40), (4, 37, 66)):
        z = fractal_bed(nx, ny, 3.0, seed=seed).astype(np.float32)
        mask = z < np.percentile(z, 70)
        mask[:3, :] = mask[-3:, :] = False
        mask[:, :3] = mask[:, -3:] = False
        s = Solver2D(Mesh2D(nx=nx, ny=ny, dx=3.0, dy=3.0, ngh=2),
                     Config(bc_x="fall", bc_y="fall", friction="manning"),
                     np.stack([np.where(mask, 0.3, 0.0), np.zeros_like(z), np.zeros_like(z)]).astype(np.float32), z)
        s.set_inside_mask(mask)
        s.set_manning_table(np.pad(voronoi_classes(nx, ny, n_seeds=8, seed=seed), 2, mode="edge"),
                            MANNING_CLASSES)
        cs = CompressedSolver.from_dense(s)
        cs.set_rain(RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[60.0, 60.0]))
        members.append(cs)
    return Ensemble(members)


def _two_steps(entry, ens, scratch=None):
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _ptr, _stream
    p0 = ens._prepare(600.0, 10 ** 9, None)
    for k in range(2):
        a = ens._args(ens._q[(p0 + k) % 2], ens._q[(p0 + k + 1) % 2])
        if scratch is not None:
            a.scratch = _ptr(scratch)
        L.call(entry, C.byref(a), _stream())
    torch.cuda.synchronize()
    return p0


def test_static_scratch_step_matches_caller_scratch_step():
    ref, stat = _ensemble(), _ensemble()
    p_ref = _two_steps("gsw_ensemble_step", ref)
    sentinel = torch.full((4,), 7, dtype=torch.int32, device="cuda")
    p_st = _two_steps("gsw_ensemble_step_static", stat, scratch=sentinel)
    assert p_ref == p_st
    assert bytes(ref.read_states()) == bytes(stat.read_states())
    for c in range(3):
        assert same(ref._q[p_ref][c].cpu().numpy(), stat._q[p_st][c].cpu().numpy())
    assert sentinel.cpu().tolist() == [7, 7, 7, 7]      # the caller's scratch is not used
    sts = stat.read_states()
    assert all(int(sts[k].steps) == 2 and sts[k].pending == 1 for k in range(2))
    # a second pair of calls continues from the left-at-zero ticket
    _two_steps("gsw_ensemble_step", ref)
    _two_steps("gsw_ensemble_step_static", stat)
    assert bytes(ref.read_states()) == bytes(stat.read_states())


def _loop_without_scratch(ens, n_steps):
    """The ensemble loop a host with no allocator runs: the initial wave speed, the dt
    rule and the static-scratch step, every call with a NULL scratch pointer."""
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _stream
    ens._build_members(600.0, 10 ** 9, None)
    ens._all_done.zero_()
    q = ens._q
    for entry in ("gsw_ensemble_lammax", "gsw_ensemble_finalize"):
        a = ens._args(q[0], q[0])
        a.scratch = None
        L.call(entry, C.byref(a), _stream())
    for k in range(n_steps):
        a = ens._args(q[k % 2], q[(k + 1) % 2])
        a.scratch = None
        L.call("gsw_ensemble_step_static", C.byref(a), _stream())
    torch.cuda.synchronize()


def test_whole_loop_runs_without_caller_scratch():
    """lammax, finalize and the static step with scratch = NULL give the same states and
    fields as the caller-scratch loop, over several steps (the static words start and end
    each step at zero)."""
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _stream
    ref, stat = _ensemble(), _ensemble()
    p0 = ref._prepare(600.0, 10 ** 9, None)
    assert p0 == 0
    n = 5
    for k in range(n):
        L.call("gsw_ensemble_step", C.byref(ref._args(ref._q[k % 2], ref._q[(k + 1) % 2])), _stream())
    torch.cuda.synchronize()
    _loop_without_scratch(stat, n)
    assert bytes(ref.read_states()) == bytes(stat.read_states())
    for c in range(3):
        assert same(ref._q[n % 2][c].cpu().numpy(), stat._q[n % 2][c].cpu().numpy())
    sts = stat.read_states()
    assert all(int(sts[k].steps) == n for k in range(2))
