"""The C ABI library loads here (no GPU) and exports every entry point include/gsw.h
declares; the ctypes layouts match the C structs."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    txt = (ROOT / "include" / "gsw.h").read_text()
    return sorted(set(re.findall(r"GSW_API\s+[\w\s\*]+?\b(gsw_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = _declared()
    assert "gsw_dense_step" in names and "gsw_dt_finalize" in names and len(names) >= 10


def test_library_loads_and_exports_all_declared():
    from geoswe_b200 import _lib
    L = _lib.lib()
    for n in _declared():
        assert hasattr(L, n), n
    assert L.gsw_abi_version() == _lib.ABI_VERSION
    assert set(_declared()) == set(_lib.exported_symbols())


def test_struct_layouts_match_c(tmp_path):
    from geoswe_b200 import _lib
    src = tmp_path / "abi.c"
    checks = {"GswLoopState": ["lam_bits", "dt_f32", "done", "reserved"],
              "GswDtParams": ["cfl_dmin", "max_steps", "rain_lim", "n_rain"],
              "GswDenseArgs": ["pitch", "state", "lam_target", "rain", "n_cls_pitch", "n_field", "vcap",
                               "max_h", "cfl_skip", "h_cfl", "warps"],
              "GswBcArgs": ["pitch", "kinds", "state"],
              "GswStageArgs": ["pitch", "bed_is_f32", "time_s", "lam_target", "g", "h_cfl"],
              "GswInflowArgs": ["pitch", "step_off", "nx_n", "t_knots", "state", "hsum"],
              "GswFlatInflowArgs": ["n_knots", "nx_n", "t_knots", "state", "hsum", "dry"],
              "GswFlatArgs": ["n_bricks", "flags", "bed", "inv_dx", "h_min_cfl", "linf", "state", "rain",
                              "ny", "n_tab_len", "vcap", "keep_h", "max_h", "warps", "segments", "brick_lo",
                              "brick_hi"],
              "GswMember": ["dt", "inv_dx", "vcap", "linf", "rain_kind", "rain", "n_tab"],
              "GswEnsembleArgs": ["n_bricks", "n_members", "grid", "brick_ij", "flags", "q0", "bed",
                                  "members", "states", "scratch", "all_done", "run", "lean"],
              "GswSeamArgs": ["q0", "nslots", "slot", "pos", "n", "dense", "stride", "scatter", "reserved"]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT}/include/gsw.h"', "int main(){"]
    for s, fs in checks.items():
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fs:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.strip().splitlines():
        key, val = line.rsplit(" ", 1)
        if "." in key:
            cls, f = key.split(".")
            got = getattr(getattr(_lib, cls), f).offset
        else:
            got = C.sizeof(getattr(_lib, key))
        assert got == int(val), (key, got, val)


def test_solver_refuses_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    import numpy as np
    from geoswe_b200 import Config, Mesh2D, Solver2D
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        Solver2D(Mesh2D(8, 8, 1.0, 1.0, ngh=2), Config(), np.zeros((3, 8, 8)), np.zeros((8, 8)))


@pytest.mark.parametrize("lo,hi", [(5, 11), (-1, 3), (6, 4)])
def test_flat_step_refuses_a_brick_range_outside_the_bricks(lo, hi):
    """The argument checks of gsw_flat_step run before any device call: a brick range
    outside [0, n_bricks) is refused with GSW_ERR_INVALID and a message."""
    from geoswe_b200 import _lib as L
    a = L.GswFlatArgs()
    a.abi_version = L.ABI_VERSION
    a.dtype = L.F32
    a.brick_h, a.n_bricks, a.warps, a.segments = 16, 10, 4, 1
    fake = C.c_void_p(0x1000)                 # never dereferenced: the call returns first
    a.brick_ij = a.brick_nbr = a.flags = fake
    a.q0 = a.q1 = a.q2 = a.qn0 = a.qn1 = a.qn2 = a.bed = fake
    a.inv_dx = a.inv_dy = 1.0
    a.g, a.h_min, a.h_min_cfl = 9.81, 1e-6, 1e-6
    a.state, a.n_tab, a.n_tab_len = fake, fake, 1
    a.brick_lo, a.brick_hi = lo, hi
    lib = L.lib()
    rc = lib.gsw_flat_step(C.byref(a), None)
    assert rc == L.ERR_INVALID
    assert b"brick range" in lib.gsw_last_error()


@pytest.mark.parametrize("h_min,h_cfl", [(0.0, 1e-6), (1e-6, 0.0), (-1e-6, 1e-6), (float("nan"), 1e-6)])
def test_step_refuses_a_divisor_floor_that_is_not_positive(h_min, h_cfl):
    """h_min and the wave speed's h_cfl floor the step's divisors, so the dense and flat
    steps refuse a value that is not > 0 (before any device call)."""
    from geoswe_b200 import _lib as L
    lib = L.lib()
    fake = C.c_void_p(0x1000)                 # never dereferenced: the call returns first
    d = L.GswDenseArgs()
    d.abi_version, d.dtype = L.ABI_VERSION, L.F32
    d.nxp = d.nyp = d.pitch = 16
    d.ngh, d.tile_rows, d.warps = 2, 4, 4
    d.q0 = d.q1 = d.q2 = d.qn0 = d.qn1 = d.qn2 = d.bed = d.state = fake
    d.inv_dx = d.inv_dy = 1.0
    d.g, d.h_min, d.h_cfl = 9.81, h_min, h_cfl
    assert lib.gsw_dense_step(C.byref(d), None) == L.ERR_INVALID
    assert b"must be > 0" in lib.gsw_last_error()
    f = L.GswFlatArgs()
    f.abi_version, f.dtype = L.ABI_VERSION, L.F32
    f.brick_h, f.n_bricks, f.warps, f.segments = 16, 4, 4, 1
    f.brick_ij = f.brick_nbr = f.flags = fake
    f.q0 = f.q1 = f.q2 = f.qn0 = f.qn1 = f.qn2 = f.bed = f.state = f.n_tab = fake
    f.n_tab_len = 1
    f.inv_dx = f.inv_dy = 1.0
    f.g, f.h_min, f.h_min_cfl = 9.81, h_min, h_cfl
    assert lib.gsw_flat_step(C.byref(f), None) == L.ERR_INVALID
    assert b"must be > 0" in lib.gsw_last_error()
