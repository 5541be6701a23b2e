"""ctypes binding of libgsw.so (include/gsw.h).

The library is the product's only compute path: if it is missing or fails to load,
importing a solver raises. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgsw.so"

ABI_VERSION = 4

OK = 0
ERR_INVALID, ERR_CUDA, ERR_ABI, ERR_NONFINITE, ERR_RANGE, ERR_TIMEOUT = -1, -2, -3, -4, -5, -6

F32, F64 = 0, 1
BC_EXTRAPOLATE, BC_WALL, BC_FALL, BC_PERIODIC, BC_NONE = 0, 1, 2, 3, 4
BC_CODES = {"extrapolate": BC_EXTRAPOLATE, "wall": BC_WALL, "fall": BC_FALL,
            "periodic": BC_PERIODIC, "none": BC_NONE}
RAIN_NONE, RAIN_UNIFORM, RAIN_GRIDDED, RAIN_LOOKUP = 0, 1, 2, 3
ARITH_EXACT, ARITH_FAST, ARITH_PORTABLE = 0, 1, 2
ARITH_CODES = {"exact": ARITH_EXACT, "fast": ARITH_FAST, "portable": ARITH_PORTABLE}
FRICTION_NONE, FRICTION_TABLE, FRICTION_FIELD = 0, 1, 2
NORM_LINF, NORM_L2 = 0, 1
BRICK_W, BRICK_PITCH = 30, 32

vp = C.c_void_p
i32, i64, u32, u64, f64 = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_double


class GswLoopState(C.Structure):
    _fields_ = [("t", f64), ("dt", f64), ("t_new", f64), ("steps", i64), ("lam_bits", u64),
                ("lam_used", f64), ("dt_f32", C.c_float), ("rain_idx", i32), ("done", i32),
                ("error", i32), ("pending", i32), ("reserved", i32 * 3)]


class GswDtParams(C.Structure):
    _fields_ = [("abi_version", u32), ("mode", i32), ("cfl_dmin", f64), ("lam_floor", f64),
                ("t_end", f64), ("eps_end", f64), ("dt_max", f64), ("fixed_dt", f64),
                ("max_steps", i64), ("rain_t", vp), ("rain_lim", vp), ("n_rain", i32),
                ("clip_flat", i32), ("dt_table", vp), ("dt_log", vp)]


class GswDenseArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("nxp", i32), ("nyp", i32), ("ngh", i32),
                ("pitch", i64),
                ("q0", vp), ("q1", vp), ("q2", vp), ("qn0", vp), ("qn1", vp), ("qn2", vp),
                ("bed", vp), ("inside_mask", vp), ("mask_pitch", i64),
                ("inv_dx", f64), ("inv_dy", f64), ("g", f64), ("h_min", f64),
                ("state", vp), ("lam_target", vp), ("rain_kind", i32), ("rain", vp),
                ("friction_kind", i32), ("n_cls", vp), ("n_cls_pitch", i64), ("n_tab", vp),
                ("n_tab_len", i32), ("n_field", vp), ("vcap", f64), ("quadratic", i32),
                ("keep_h", i32), ("max_h", vp), ("cfl_skip", vp), ("h_cfl", f64),
                ("tile_rows", i32), ("warps", i32), ("min_blocks", i32), ("arith", i32),
                ("row_lo", i32), ("row_hi", i32), ("col_lo", i32), ("col_hi", i32)]


class GswBcArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("nxp", i32), ("nyp", i32), ("ngh", i32),
                ("pitch", i64), ("q0", vp), ("q1", vp), ("q2", vp), ("kinds", i32 * 4),
                ("state", vp)]


class GswStageArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("pitch", i64), ("q0", vp), ("q1", vp),
                ("q2", vp), ("cell_off", vp), ("bed64", vp), ("bed_is_f32", i32), ("n_cells", i32),
                ("time_s", vp), ("stage_m", vp), ("n_knots", i32), ("state", vp),
                ("lam_target", vp), ("cfl_ghost", vp), ("g", f64), ("h_cfl", f64)]


class GswInflowArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("pitch", i64), ("q0", vp), ("q1", vp),
                ("q2", vp), ("bed", vp), ("inlet_off", vp), ("n", i32), ("ngh", i32),
                ("step_off", i64), ("nx_n", f64), ("ny_n", f64), ("ds", f64), ("dry_frac", f64),
                ("t_knots", vp), ("q_knots", vp), ("n_knots", i32), ("state", vp), ("hsum", vp)]


class GswFlatArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("brick_h", i32), ("warps", i32), ("min_blocks", i32),
                ("arith", i32), ("n_bricks", i64),
                ("brick_ij", vp), ("brick_nbr", vp), ("flags", vp),
                ("q0", vp), ("q1", vp), ("q2", vp), ("qn0", vp), ("qn1", vp), ("qn2", vp), ("bed", vp),
                ("inv_dx", f64), ("inv_dy", f64), ("g", f64), ("h_min", f64), ("h_min_cfl", f64),
                ("linf", i32), ("rain_kind", i32), ("state", vp), ("lam_target", vp), ("rain", vp),
                ("ngh", i32), ("nx", i32), ("ny", i32), ("n_tab_len", i32), ("n_cls", vp), ("n_tab", vp),
                ("vcap", f64), ("quadratic", i32), ("keep_h", i32), ("max_h", vp), ("rain_lookup", vp),
                ("rain_ncol", i32), ("segments", i32), ("brick_lo", C.c_int64), ("brick_hi", C.c_int64)]


class GswFlatInflowArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("q0", vp), ("q1", vp), ("q2", vp), ("bed", vp),
                ("ghost_slot", vp), ("nbr_slot", vp), ("n", i32), ("n_knots", i32), ("nx_n", f64),
                ("ny_n", f64), ("ds", f64), ("t_knots", vp), ("q_knots", vp), ("state", vp), ("hsum", vp),
                ("dry", vp)]


class GswFlatAdjArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("min_blocks", i32), ("f", GswFlatArgs),
                ("lam_in0", vp), ("lam_in1", vp), ("lam_in2", vp), ("lam_out0", vp), ("lam_out1", vp),
                ("lam_out2", vp), ("rbar0", vp), ("rbar1", vp), ("rbar2", vp), ("n_bar", vp), ("rate_bar", vp)]


class GswGaugeArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("q0", vp), ("slots", vp), ("n", i32), ("offset", i32),
                ("first", i64), ("count", i64), ("series", vp), ("target", vp), ("weight", f64), ("lam0", vp),
                ("state", vp)]


class GswFlatRingArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("q0", vp), ("q1", vp), ("q2", vp), ("slots", vp),
                ("bed", vp), ("wg", vp), ("n", i32), ("NG", i32), ("t_common", vp), ("n_t", i32),
                ("reserved0", i32), ("stage_all", vp), ("state", vp)]


class GswFlatForcingArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("phase", i32), ("q0", vp), ("q1", vp), ("q2", vp), ("flags", vp),
                ("nslots", i64), ("h_min", C.c_float), ("reserved0", i32), ("state", vp), ("n_cls", vp),
                ("infil_tab", vp), ("sp_slots", vp), ("sp_keep", vp), ("sp_amb", vp), ("sp_n", i32),
                ("ga_mode", i32), ("ga_cls", vp), ("Ks_t", vp), ("psi_t", vp), ("dth_t", vp), ("F", vp),
                ("Fmax", vp), ("inv_tau", vp), ("cl_slots", vp), ("cl_hmax", vp), ("cl_n", i32), ("dr_n", i32),
                ("dr_slots", vp), ("dr_htgt", vp)]


class GswSeamArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("dtype", i32), ("q0", vp), ("q1", vp), ("q2", vp), ("nslots", i64),
                ("slot", vp), ("pos", vp), ("n", i64), ("dense", vp), ("stride", i64), ("scatter", i32),
                ("reserved", i32)]


class GswMember(C.Structure):
    _fields_ = [("dt", GswDtParams), ("inv_dx", C.c_float), ("g", C.c_float), ("h_min", C.c_float),
                ("h_min_cfl", C.c_float), ("vcap", C.c_float), ("linf", i32), ("quadratic", i32),
                ("keep_h", i32), ("rain_kind", i32), ("g_recip", C.c_float), ("rain", vp), ("n_tab", vp)]


class GswTuneResult(C.Structure):
    _fields_ = [("abi_version", u32), ("tile_rows", i32), ("warps", i32), ("min_blocks", i32),
                ("segments", i32), ("n_tried", i32), ("ms", C.c_float), ("reserved", i32)]


class GswEnsembleArgs(C.Structure):
    _fields_ = [("abi_version", u32), ("brick_h", i32), ("n_bricks", i64), ("n_members", i32),
                ("warps", i32), ("grid", i32), ("min_blocks", i32), ("arith", i32), ("segments", i32),
                ("brick_ij", vp), ("brick_nbr", vp),
                ("brick_member", vp), ("flags", vp), ("n_cls", vp), ("q0", vp), ("q1", vp), ("q2", vp),
                ("qn0", vp), ("qn1", vp), ("qn2", vp), ("bed", vp), ("max_h", vp), ("members", vp),
                ("states", vp), ("scratch", vp), ("all_done", vp), ("member_brick_off", vp), ("run", vp), ("lean", i32)]


# entry point -> argtypes
_PROTOS = {
    "gsw_dense_step": [C.POINTER(GswDenseArgs), vp],
    "gsw_dense_rhs": [C.POINTER(GswDenseArgs), vp],
    "gsw_dense_lammax": [C.POINTER(GswDenseArgs), vp, vp],
    "gsw_bc_fill": [C.POINTER(GswBcArgs), vp],
    "gsw_stage_apply": [C.POINTER(GswStageArgs), vp],
    "gsw_lam_cells": [C.POINTER(GswStageArgs), vp],
    "gsw_inflow_apply": [C.POINTER(GswInflowArgs), vp],
    "gsw_inflow_depth_sum": [C.POINTER(GswInflowArgs), vp, vp],
    "gsw_dt_finalize": [C.POINTER(GswDtParams), vp, vp],
    "gsw_dt_params_upload": [C.POINTER(GswDtParams), vp, vp],
    "gsw_dense_autotune": [C.POINTER(GswDenseArgs), C.c_int32, C.c_int32, C.POINTER(GswTuneResult), vp],
    "gsw_flat_autotune": [C.POINTER(GswFlatArgs), C.c_int32, C.c_int32, C.POINTER(GswTuneResult), vp],
    "gsw_dt_finalize_dev": [vp, vp, vp],
    "gsw_loop_commit": [vp, vp],
    "gsw_flat_inflow_apply": [C.POINTER(GswFlatInflowArgs), vp],
    "gsw_flat_inflow_depth_sum": [C.POINTER(GswFlatInflowArgs), vp, vp],
    "gsw_flat_forcings": [C.POINTER(GswFlatForcingArgs), vp],
    "gsw_flat_ring_stage": [C.POINTER(GswFlatRingArgs), vp],
    "gsw_seam_copy": [C.POINTER(GswSeamArgs), vp],
    "gsw_adj_flat_step": [C.POINTER(GswFlatAdjArgs), vp],
    "gsw_adj_flat_inflow": [C.POINTER(GswFlatInflowArgs), vp, vp, vp, vp, vp],
    "gsw_gauge_record": [C.POINTER(GswGaugeArgs), vp],
    "gsw_gauge_adjoint": [C.POINTER(GswGaugeArgs), vp],
    "gsw_flat_step": [C.POINTER(GswFlatArgs), vp],
    "gsw_flat_rhs": [C.POINTER(GswFlatArgs), vp],
    "gsw_flat_lammax": [C.POINTER(GswFlatArgs), vp, vp],
    "gsw_mesh_count": [vp, C.c_int, C.c_int, C.c_int, vp, vp],
    "gsw_mesh_build": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp],
    "gsw_bricks_build": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp],
    "gsw_bricks_slot_of": [vp, C.c_int64, vp, C.c_int64, C.c_int, C.c_int, C.c_int, vp],
    "gsw_div_const_recip": [C.c_float],
    "gsw_ensemble_lammax": [C.POINTER(GswEnsembleArgs), vp],
    "gsw_ensemble_finalize": [C.POINTER(GswEnsembleArgs), vp],
    "gsw_ensemble_step": [C.POINTER(GswEnsembleArgs), vp],
    "gsw_ensemble_step_static": [C.POINTER(GswEnsembleArgs), vp],
}


class GswError(RuntimeError):
    """A libgsw entry point returned a non-zero status."""

    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed ({code}): {msg}")
        self.code = code


_lib = None


def lib():
    """Load libgsw.so (once). Raises ImportError if it is missing or unloadable."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m geoswe_b200.build` "
            f"(nvcc, sm_100a). geoswe_b200 has no CPU fallback.")
    L = C.CDLL(str(LIB_PATH))
    for name, argt in _PROTOS.items():
        fn = getattr(L, name)
        fn.argtypes = argt
        fn.restype = C.c_int
    L.gsw_div_const_recip.restype = C.c_float
    L.gsw_last_error.restype = C.c_char_p
    L.gsw_last_error.argtypes = []
    L.gsw_abi_version.restype = C.c_uint32
    L.gsw_launch_count.restype = C.c_uint64
    if L.gsw_abi_version() != ABI_VERSION:
        raise ImportError(f"libgsw ABI {L.gsw_abi_version()} != {ABI_VERSION}; rebuild it")
    _lib = L
    return L


def call(name, *args):
    L = lib()
    rc = getattr(L, name)(*args)
    if rc != OK:
        raise GswError(name, rc, L.gsw_last_error().decode(errors="replace"))
    return rc


def launch_count() -> int:
    return int(lib().gsw_launch_count())


def exported_symbols():
    """Names the header declares (used by the load test)."""
    return list(_PROTOS) + ["gsw_last_error", "gsw_abi_version", "gsw_launch_count"]
