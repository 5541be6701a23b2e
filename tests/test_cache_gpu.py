"""The reference's flat-mesh cache format and checkpoints on the GPU. The golden cache
in tests/golden/reference_cache/ was written by the reference's own save_cache
(tests/golden/make_golden.py): a wet state, three Manning classes, a two-column rain
table with a per-cell lookup and a two-gauge ring stage. CompressedSolver.from_cache
loads it, runs it bit for bit as the oracle's restatement of the flat loop does on the
cache's arrays (with the oracle's portable Manning power), writes it back in the same format, and a run interrupted and resumed
from a checkpoint equals the uninterrupted run."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from tests._cases import same

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CACHE = Path(__file__).resolve().parent / "golden" / "reference_cache"


def _ld(name):
    return np.load(CACHE / (name + ".npy"))


def _oracle_from_cache():
    meta = json.load(open(CACHE / "meta.json"))
    q = [_ld(f"q{c}").astype(np.float32) for c in range(3)]
    o = oracle.OracleFlat(_ld("nbr"), _ld("is_active"), q, _ld("bed_f"), meta["dx"], ncls=_ld("mcls_f"),
                          ntab=_ld("m_tab"), rain_times=_ld("rain_t_s"),
                          rain_table=_ld("rain_native_rate_dev").astype(np.float32),
                          rain_lookup=_ld("rain_lookup_flat").astype(np.int64))
    n, NG = meta["ring_n"], meta["ring_NG"]
    o.set_ring(_ld("ring_rflat").astype(np.int64), _ld("ring_rbed"), _ld("ring_rwg").reshape(n, NG),
               _ld("ring_t_common"), _ld("ring_stage_all"))
    return o


def test_from_cache_tables_state_and_run_bitwise():
    from geoswe_b200.compressed import CompressedSolver
    cs = CompressedSolver.from_cache(CACHE, arith="portable")     # the oracle's Manning power
    assert np.array_equal(cs.nbr, _ld("nbr")) and np.array_equal(cs.is_active, _ld("is_active"))
    assert np.array_equal(cs.ij_active, _ld("ij_active"))
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), _ld(f"q{c}"))
    o = _oracle_from_cache()
    n_g = cs.run(t_end=500.0)
    n_o = o.run(t_end=500.0)
    assert n_g == n_o and n_g > 20
    assert cs.t == o.t
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), o.q[c]), c


def test_save_cache_round_trip(tmp_path):
    from geoswe_b200.compressed import CompressedSolver
    cs = CompressedSolver.from_cache(CACHE)
    cs.save_cache(tmp_path)
    meta = json.load(open(tmp_path / "meta.json"))
    ref = json.load(open(CACHE / "meta.json"))
    for k in ("nxp", "nyp", "ngh", "dx", "N", "has_ring", "has_rain", "ring_NG", "ring_n"):
        assert meta[k] == ref[k], k
    for name in ("nbr", "is_active", "ij_active", "q0", "q1", "q2", "bed_f", "mcls_f", "m_tab",
                 "rain_native_rate_dev", "rain_lookup_flat", "rain_t_s", "ring_rflat", "ring_rbed", "ring_rwg",
                 "ring_t_common", "ring_stage_all"):
        a, b = np.load(tmp_path / (name + ".npy")), _ld(name)
        assert np.array_equal(a.reshape(-1).astype(np.float64), b.reshape(-1).astype(np.float64)), name
    cs2 = CompressedSolver.from_cache(tmp_path)
    cs.run(t_end=300.0)
    cs2.run(t_end=300.0)
    for c in range(3):
        assert same(cs.flat(c).cpu().numpy(), cs2.flat(c).cpu().numpy())


def test_checkpoint_resume_equals_uninterrupted(tmp_path):
    from geoswe_b200.compressed import CompressedSolver
    t_end = 700.0
    full = CompressedSolver.from_cache(CACHE)
    n_full = full.run(t_end=t_end, window=8, checkpoint_every_s=150.0, ckpt_dir=tmp_path / "a")
    meta = json.load(open(tmp_path / "a" / "ckpt_meta.json"))
    assert meta["t"] == full.t and meta["steps"] == n_full
    # an interrupted run: stopped by a step cap (no clipped step), checkpointed on the way
    part = CompressedSolver.from_cache(CACHE)
    m = n_full // 3
    part.run(t_end=t_end, window=8, max_steps=m, checkpoint_every_s=150.0, ckpt_dir=tmp_path / "b")
    resumed = CompressedSolver.from_cache(CACHE)
    n_rest = resumed.run(t_end=t_end, window=8, resume=True, ckpt_dir=tmp_path / "b")
    assert resumed.nsteps == n_full and m + n_rest == n_full
    assert resumed.t == full.t
    for c in range(3):
        assert same(resumed.flat(c).cpu().numpy(), full.flat(c).cpu().numpy())
