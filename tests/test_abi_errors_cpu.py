"""The library's argument checks, on the CPU: each call below is refused before any
CUDA work (so no GPU is needed), with the documented code and a message."""
import ctypes as C

import pytest

from geoswe_b200 import _lib as L


def _call(name, *args):
    lib = L.lib()
    rc = getattr(lib, name)(*args)
    return rc, lib.gsw_last_error().decode()


def _dense(**kw):
    a = L.GswDenseArgs()
    a.abi_version = L.ABI_VERSION
    a.dtype = L.F32
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def test_abi_version_is_checked():
    rc, msg = _call("gsw_dense_step", C.byref(_dense(abi_version=L.ABI_VERSION + 1)), None)
    assert rc == L.ERR_ABI and "abi_version" in msg


def test_fast_arithmetic_is_binary32_only():
    rc, msg = _call("gsw_dense_step", C.byref(_dense(dtype=L.F64, arith=L.ARITH_FAST)), None)
    assert rc == L.ERR_INVALID and "binary32" in msg
    rc, msg = _call("gsw_dense_step", C.byref(_dense(arith=7)), None)
    assert rc == L.ERR_INVALID and "arith" in msg
    f = L.GswFlatArgs()
    f.abi_version, f.dtype, f.arith = L.ABI_VERSION, L.F64, L.ARITH_FAST
    rc, msg = _call("gsw_flat_step", C.byref(f), None)
    assert rc == L.ERR_INVALID and "binary32" in msg


def test_dense_shape_checks():
    rc, msg = _call("gsw_dense_step", C.byref(_dense(nxp=4, nyp=4, ngh=2)), None)
    assert rc == L.ERR_INVALID and "ngh" in msg


def test_dt_params_are_checked_on_the_host():
    p = L.GswDtParams()
    p.abi_version = L.ABI_VERSION
    p.mode, p.cfl_dmin = 0, 0.0
    rc, msg = _call("gsw_dt_params_upload", C.byref(p), C.c_void_p(16), None)
    assert rc == L.ERR_INVALID and "cfl_dmin" in msg
    p.mode, p.fixed_dt = 1, 0.0
    rc, msg = _call("gsw_dt_params_upload", C.byref(p), C.c_void_p(16), None)
    assert rc == L.ERR_INVALID and "fixed_dt" in msg
    p.mode = 2
    rc, msg = _call("gsw_dt_params_upload", C.byref(p), C.c_void_p(16), None)
    assert rc == L.ERR_INVALID and "dt_table" in msg
    p.mode, p.cfl_dmin = 0, 1.0
    rc, msg = _call("gsw_dt_params_upload", C.byref(p), None, None)
    assert rc == L.ERR_INVALID and "destination" in msg


def test_ensemble_and_autotune_checks():
    e = L.GswEnsembleArgs()
    e.abi_version = L.ABI_VERSION
    rc, msg = _call("gsw_ensemble_step", C.byref(e), None)
    assert rc == L.ERR_INVALID
    r = L.GswTuneResult()
    r.abi_version = L.ABI_VERSION
    rc, msg = _call("gsw_dense_autotune", C.byref(_dense()), 0, 0, C.byref(r), None)
    assert rc == L.ERR_INVALID and "reps" in msg
    r.abi_version = 0
    rc, msg = _call("gsw_dense_autotune", C.byref(_dense()), 2, 0, C.byref(r), None)
    assert rc == L.ERR_ABI


def test_adjoint_refuses_fast_arguments():
    a = L.GswFlatAdjArgs()
    a.abi_version = L.ABI_VERSION
    a.f.abi_version = L.ABI_VERSION
    a.min_blocks = 3
    rc, msg = _call("gsw_adj_flat_step", C.byref(a), None)
    assert rc == L.ERR_INVALID


def test_constant_reciprocal_check():
    """gsw_div_const_recip: RN(1/g) for the gravity values in use (their sequence is
    exhaustively checked to give the IEEE quotient), 0 for values it cannot take."""
    import numpy as np
    lib = L.lib()
    for g in (9.81, 9.80665, 9.8):
        y = lib.gsw_div_const_recip(g)
        assert y == float(np.float32(1.0 / np.float64(np.float32(g))))
    assert lib.gsw_div_const_recip(0.0) == 0.0
    assert lib.gsw_div_const_recip(-9.81) == 0.0
    assert lib.gsw_div_const_recip(float("inf")) == 0.0


def test_seam_copy_checks():
    a = L.GswSeamArgs()
    a.abi_version, a.dtype, a.n, a.stride = L.ABI_VERSION, L.F32, 0, 8
    assert _call("gsw_seam_copy", C.byref(a), None)[0] == L.OK            # nothing to move
    a.n = 4
    rc, msg = _call("gsw_seam_copy", C.byref(a), None)
    assert rc == L.ERR_INVALID and "null" in msg
    a.stride = 0
    rc, msg = _call("gsw_seam_copy", C.byref(a), None)
    assert rc == L.ERR_INVALID and "stride" in msg


def test_dense_window_is_checked():
    """A window reaching outside the computed range (or empty) is refused before any
    launch."""
    fake = C.c_void_p(256)
    for w in [(1, 5, 0, 0), (2, 19, 0, 0), (6, 6, 0, 0), (0, 0, 3, 2)]:
        a = _dense(nxp=20, nyp=20, ngh=2, pitch=32, q0=fake, q1=fake, q2=fake, qn0=fake, qn1=fake, qn2=fake,
                   bed=fake, row_lo=w[0], row_hi=w[1], col_lo=w[2], col_hi=w[3])
        rc, msg = _call("gsw_dense_step", C.byref(a), None)
        assert rc == L.ERR_INVALID and "window" in msg, (w, rc, msg)
