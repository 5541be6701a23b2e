"""Compressed-mesh tables, bit-exact against the reference's CompressedSWE
(tests/golden/reference_mesh.npz, produced by the reference itself), and the brick
layout's bookkeeping. Host code only (no GPU)."""
from pathlib import Path

import numpy as np
import pytest

from geoswe_b200.compressed import BRICK_W, build_bricks, build_tables
from geoswe_b200.synthetic import dilate_cross

M = np.load(Path(__file__).resolve().parent / "golden" / "reference_mesh.npz")
CASES = sorted({k.split("_")[1] for k in M.files})


@pytest.mark.parametrize("case", CASES)
def test_tables_bit_exact(case):
    """Every case the reference builds (including one inside cell, and inside cells on
    the array edge whose ring is not covered) is matched bit for bit; a case the
    reference refuses (no inside cell) is refused here with the same ValueError."""
    if f"mesh_{case}_raises" in M.files:
        assert "no interior neighbors" in str(M[f"mesh_{case}_raises"])
        with pytest.raises(ValueError, match="no interior neighbors"):
            build_tables(M[f"mesh_{case}_inside"], ring=2)
        return
    tb = build_tables(M[f"mesh_{case}_inside"], ring=2)
    assert np.array_equal(tb["ij"], M[f"mesh_{case}_ij"])
    assert np.array_equal(tb["active_id"], M[f"mesh_{case}_aid"])
    assert np.array_equal(tb["nbr"], M[f"mesh_{case}_nbr16"])
    assert tb["nbr"].dtype == np.int16
    assert np.array_equal(tb["is_active"], M[f"mesh_{case}_active"])
    assert tb["fully_covered"] == bool(M[f"mesh_{case}_covered"])


def test_int16_overflow_refused():
    inside = np.zeros((6, 33000), np.uint8)
    inside[2:4, 2:-2] = 1
    with pytest.raises(ValueError, match="int16"):
        build_tables(inside, ring=2)


def test_dilation_matches_scipy():
    from scipy.ndimage import binary_dilation
    rng = np.random.default_rng(3)
    m = rng.random((57, 43)) < 0.1
    assert np.array_equal(dilate_cross(m, 2), binary_dilation(m, iterations=2))
    assert np.array_equal(dilate_cross(m, 8), binary_dilation(m, iterations=8))


@pytest.mark.parametrize("bh", [2, 8, 16])
def test_bricks_cover_stored_cells(bh):
    inside = M["mesh_blob_inside"]
    tb = build_tables(inside)
    stored = tb["active_id"] >= 0
    bij, bnbr = build_bricks(stored, bh)
    nb = len(bij)
    # every stored cell's brick exists, bricks are unique, links are consistent
    keys = set(map(tuple, bij.tolist()))
    assert len(keys) == nb
    for i, j in np.argwhere(stored):
        assert (i // bh, j // BRICK_W) in keys
    idx = {tuple(k): n for n, k in enumerate(bij.tolist())}
    for n, (a, c) in enumerate(bij.tolist()):
        for d, (da, dc) in enumerate([(-1, 0), (1, 0), (0, -1), (0, 1)]):
            exp = idx.get((a + da, c + dc), nb)
            assert bnbr[n, d] == exp


def test_reference_cache_tables_match_builder():
    """The golden cache written by the reference's save_cache holds the canonical tables
    this package's host builder produces for the same active set."""
    import json
    from pathlib import Path
    from geoswe_b200.compressed import build_tables
    d = Path(__file__).resolve().parent / "golden" / "reference_cache"
    meta = json.load(open(d / "meta.json"))
    ij = np.load(d / "ij_active.npy")
    act = np.load(d / "is_active.npy")
    inside = np.zeros((meta["nxp"], meta["nyp"]), np.uint8)
    inside[ij[act != 0, 0], ij[act != 0, 1]] = 1
    t = build_tables(inside, ring=2)
    assert t["N"] == meta["N"]
    assert np.array_equal(t["ij"], ij) and np.array_equal(t["nbr"], np.load(d / "nbr.npy"))
    assert np.array_equal(t["is_active"], act)


@pytest.mark.parametrize("bh", [4, 16])
def test_bricks_slot_of(bh):
    """gsw_bricks_slot_of places every canonical cell in its brick, at its row and
    column, each in its own slot."""
    import ctypes as C
    from geoswe_b200 import _lib as L
    inside = M["mesh_band_inside"]
    tb = build_tables(inside)
    stored = tb["active_id"] >= 0
    bij, _ = build_bricks(stored, bh)
    nxp, nyp = inside.shape
    ij = np.ascontiguousarray(tb["ij"], np.int32)
    slot = np.empty(len(ij), np.int64)
    lib = L.lib()
    rc = lib.gsw_bricks_slot_of(ij.ctypes.data, len(ij), np.ascontiguousarray(bij, np.int32).ctypes.data, len(bij),
                                bh, nxp, nyp, slot.ctypes.data)
    assert rc == 0, lib.gsw_last_error()
    BS = bh * 32
    assert len(np.unique(slot)) == len(slot) and slot.min() >= 0 and slot.max() < len(bij) * BS
    b, rem = slot // BS, slot % BS
    assert np.array_equal(bij[b, 0] * bh + rem // 32, ij[:, 0])
    assert np.array_equal(bij[b, 1] * BRICK_W + rem % 32, ij[:, 1])
    bad = ij.copy()
    bad[0] = (nxp + 5, 0)
    assert lib.gsw_bricks_slot_of(bad.ctypes.data, len(bad), np.ascontiguousarray(bij, np.int32).ctypes.data,
                                  len(bij), bh, nxp, nyp, slot.ctypes.data) == L.ERR_INVALID
