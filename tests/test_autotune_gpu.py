"""Launch-shape search: the Python tuner (geoswe_b200.autotune) and the library's own
(gsw_dense_autotune, gsw_flat_autotune). A winner is one of the candidates, is cached,
leaves the solver's state alone, and -- like every launch shape -- changes no bit of
the results."""
import ctypes as C
import warnings

import numpy as np
import pytest

from tests._cases import flowing, same

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def _tune_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("GSW_TUNE_CACHE", str(tmp_path / "autotune.json"))


def _dense(arith="exact", **kw):
    from geoswe_b200 import Config, Mesh2D, Solver2D
    q0, bed = flowing(70, 97, seed=11, dtype=np.float32)
    return Solver2D(Mesh2D(nx=70, ny=97, dx=2.0, dy=2.0, ngh=2),
                    Config(bc_x="wall", bc_y="wall", friction="manning", manning_n=0.03, arith=arith), q0, bed, **kw)


def _flat():
    from geoswe_b200 import Config, Mesh2D, RainfallForcing, Solver2D
    from geoswe_b200.compressed import CompressedSolver
    from geoswe_b200.synthetic import fractal_bed
    z = fractal_bed(80, 90, 3.0, seed=3).astype(np.float32)
    mask = z < np.percentile(z, 65)
    mask[:3, :] = mask[-3:, :] = False
    mask[:, :3] = mask[:, -3:] = False
    s = Solver2D(Mesh2D(nx=80, ny=90, dx=3.0, dy=3.0, ngh=2), Config(bc_x="fall", bc_y="fall", friction="manning",
                                                                   manning_n=0.03),
                 np.zeros((3, 80, 90), np.float32), z)
    s.set_inside_mask(mask)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        cs = CompressedSolver.from_dense(s)
    cs.set_rain(RainfallForcing(time_s=[0.0, 1e9], rate_mm_h=[60.0, 60.0]))
    return cs


def test_python_tuner_dense_caches_and_changes_no_bit():
    from geoswe_b200 import autotune
    s = _dense()
    s.run(t_end=1e9, max_steps=6)
    space = dict(tile_rows=(0, 8, 32), warps=(2, 4), min_blocks=(0, 4))
    best, table = autotune.tune_dense(s, reps=2, space=space)
    assert len(table) == 12 and best in table
    assert autotune.load("dense", 70 * 97) == best
    fresh = _dense()                                    # picks the cached shape
    assert (fresh._tile_rows, fresh._warps, fresh._min_blocks) == (best["tile_rows"], best["warps"],
                                                                  best["min_blocks"])
    runs = []
    for shape in ((0, 0, 0), (8, 2, 4), (32, 4, 0)):
        d = _dense(tile_rows=shape[0], warps=shape[1], min_blocks=shape[2], autotuned=False)
        n = d.run(t_end=30.0)
        runs.append((n, d.t, d.q.cpu().numpy()))
    for n, t, q in runs[1:]:
        assert n == runs[0][0] and t == runs[0][1]
        assert same(q[:, 2:-2, 2:-2], runs[0][2][:, 2:-2, 2:-2])


def test_python_tuner_flat_sets_and_caches():
    from geoswe_b200 import autotune
    cs = _flat()
    cs.run(t_end=1e9, max_steps=6)
    best, table = autotune.tune_flat(cs, reps=2, space=dict(warps=(2, 4), min_blocks=(0, 3), segments=(0, 2)))
    assert len(table) == 8 and best in table
    assert (cs.warps, cs.min_blocks, cs.segments) == (best["warps"], best["min_blocks"], best["segments"])
    assert autotune.load("flat", cs.nslots) == best


def test_library_dense_autotune_no_side_effects_and_cache():
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _stream
    s = _dense()
    s.run(t_end=1e9, max_steps=6)
    T = s._tables()
    q_before = s.q.cpu().numpy().copy()
    mx_before = s._max_h.cpu().numpy().copy()
    st = L.GswLoopState()
    st.dt, st.dt_f32 = 0.01, float(np.float32(0.01))
    state = torch.zeros(128, dtype=torch.uint8, device=s.device)
    state.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))), dtype=torch.uint8))
    scratch = torch.empty_like(s._buf[s._cur])
    a = s._dense_args(s._buf[s._cur], scratch, T)
    a.state = C.c_void_p(state.data_ptr())
    res = L.GswTuneResult()
    res.abi_version = L.ABI_VERSION
    L.call("gsw_dense_autotune", C.byref(a), 2, 0, C.byref(res), _stream())
    torch.cuda.synchronize()
    assert res.n_tried == 6 * 3 * 4 and res.ms > 0
    assert res.tile_rows in (0, 4, 8, 16, 32, 64) and res.warps in (2, 4, 8) and res.min_blocks in (0, 3, 4, 5)
    assert same(s.q.cpu().numpy(), q_before)                  # the step's input is untouched
    assert same(s._max_h.cpu().numpy(), mx_before)            # no running-max update
    assert bytes(state.cpu().numpy()[:C.sizeof(st)]) == bytes(st)   # loop state only read
    n0 = L.launch_count()
    again = L.GswTuneResult()
    again.abi_version = L.ABI_VERSION
    L.call("gsw_dense_autotune", C.byref(a), 2, 1, C.byref(again), _stream())
    assert L.launch_count() == n0                             # answered from the cache
    assert (again.tile_rows, again.warps, again.min_blocks, again.ms) == (res.tile_rows, res.warps,
                                                                          res.min_blocks, res.ms)


def test_library_flat_autotune():
    from geoswe_b200 import _lib as L
    from geoswe_b200.solver import _stream
    cs = _flat()
    cs.run(t_end=1e9, max_steps=6)
    st = L.GswLoopState()
    st.dt, st.dt_f32 = 0.01, float(np.float32(0.01))
    state = torch.zeros(128, dtype=torch.uint8, device=cs.device)
    state.copy_(torch.frombuffer(bytearray(bytes(st) + bytes(128 - C.sizeof(st))), dtype=torch.uint8))
    src = [x.clone() for x in cs._q[cs._cur]]
    dst = [torch.empty_like(x) for x in src]
    a = cs._args(src, dst)
    a.state = C.c_void_p(state.data_ptr())
    res = L.GswTuneResult()
    res.abi_version = L.ABI_VERSION
    L.call("gsw_flat_autotune", C.byref(a), 2, 0, C.byref(res), _stream())
    assert res.n_tried == 3 * 4 * 4 and res.segments in (0, 1, 2, 4)
    for c in range(3):
        assert same(src[c].cpu().numpy(), cs._q[cs._cur][c].cpu().numpy())
    done = L.GswLoopState()
    done.done = 1
    state.copy_(torch.frombuffer(bytearray(bytes(done) + bytes(128 - C.sizeof(done))), dtype=torch.uint8))
    with pytest.raises(L.GswError):
        L.call("gsw_flat_autotune", C.byref(a), 2, 0, C.byref(res), _stream())
