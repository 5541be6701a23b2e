"""Compile the reference's own dense-step CUDA kernels for sm_100a -- TEST INFRASTRUCTURE.

    python oracle/ref_build.py [--ref <reference checkout>/src]

The reference tree is taken from --ref, else from $GEOSWE_REFERENCE_SRC, else from the
standard checkout location of this build host (reference_src() below).

The reference keeps its GPU kernels as CUDA C text inside Python and assembles the
production variants at import (geoswe/rhs_cuda.py:1698-2192, geoswe/solver.py:152-205).
This recipe imports the reference package with a recording stand-in for CuPy, so the
exact text the reference would hand to NVRTC is captured, and compiles it with nvcc:

  oracle/_ref/ref_kernels.cu          the captured reference text + C launch wrappers
                                      (the dense fused step, the residual, lammax, the
                                      flat fused step + CFL and the flat lammax (L2 and
                                      Linf norms), and the flat loop's per-step forcing
                                      kernels)
  oracle/_ref/libref_fma.so           nvcc defaults (FMA contraction on, as NVRTC)
  oracle/_ref/libref_strict.so        --fmad=false (every operation rounded separately)

oracle/_ref/ is git-ignored (the reference's source is not committed) but travels to
the GPU box with the other built libraries; oracle/ref_runner.py drives the kernels
there as the reference's dense and flat solvers do. Nothing in the product uses them.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


class _Recorded:
    def __init__(self, code=None, name=None, options=()):
        self.code, self.name, self.options = code, name, tuple(options)

    def __call__(self, *a, **k):
        raise RuntimeError("recorded kernel: not runnable on the build host")


def _fake_cupy():
    cp = types.ModuleType("cupy")
    for n in dir(np):
        if not n.startswith("__"):
            try:
                setattr(cp, n, getattr(np, n))
            except Exception:
                pass
    cp.ndarray = np.ndarray
    cp.asnumpy = lambda a: np.asarray(a)
    cp.RawKernel = lambda code, name, options=(), **k: _Recorded(code, name, options)
    cp.RawModule = lambda code=None, options=(), **k: _Recorded(code, "module", options)
    cp.ElementwiseKernel = lambda *a, **k: _Recorded(None, k.get("name", "elementwise"))
    cp.ReductionKernel = lambda *a, **k: _Recorded(None, "reduction")
    cp.get_default_memory_pool = lambda: types.SimpleNamespace(free_all_blocks=lambda: None)
    cuda = types.ModuleType("cupy.cuda")
    cuda.runtime = types.SimpleNamespace(getDeviceCount=lambda: 1, is_hip=False,
                                         memGetInfo=lambda: (0, 0))
    cuda.Device = lambda *a: types.SimpleNamespace(compute_capability="100", id=0)
    cp.cuda = cuda
    sys.modules["cupy"] = cp
    sys.modules["cupy.cuda"] = cuda
    return cp


def capture(ref_src):
    """Return {kernel_name: source} of the reference's production kernels: the dense fused
    step and residual (rhs_cuda.py:2095-2192, 900-1207), lammax (solver.py:152-205), the
    flat fused step + CFL as CompressedStepper assembles it with the chained neighbour
    preamble (compressed_rhs.py:1082-1118 over :92-112, :716-748, :1027-1039; the reg2
    preambles index the same cells by arithmetic, compressed_rhs.py:867-877), in its no-sigma
    build with the L2 and the Linf wave-speed norm (compressed_solver.py:819-843), the flat
    lammax kernel used for a run's first dt (compressed_solver.py:200-244, 655-668), and
    the flat loop's per-step forcing kernels."""
    os.environ["GEOSWE_BACKEND"] = "cupy"
    for k in ("SWE_DENSE_XY", "SWE_BED_GRAD_LIMITER", "SWE_DRY_SKIP", "SWE_WETDRY_ZERO_H",
              "SWE_DENSE_MAXRREG"):
        os.environ.pop(k, None)
    _fake_cupy()
    sys.path.insert(0, str(ref_src))
    from geoswe import rhs_cuda as R
    from geoswe import solver as S
    k2d = R.build_dense_fstep2d_kernel(True, 1)                         # no sigma, keep-h
    kres = R._build_srm_hllc_ns("float", "fused_rhs_wb_srm_hllc_2d_ns_fp32")
    kres64 = R._build_srm_hllc_ns("double", "fused_rhs_wb_srm_hllc_2d_ns_fp64")
    from geoswe import compressed_solver as CS
    from geoswe import compressed_rhs as CR
    keep_h = int(CS._WETDRY_KEEP_H)
    kfl = CR.build_flat_fused_step_cfl_kernel(CR._PRE_B_FLAT, keep_h, no_sigma=True, tag="chained", linf=False)
    kfl_inf = CR.build_flat_fused_step_cfl_kernel(CR._PRE_B_FLAT, keep_h, no_sigma=True, tag="chained", linf=True)
    # the Linf lammax is the reference's own rewrite of its L2 text (compressed_solver.py:664-666),
    # renamed so both live in one module
    lam_inf = CS._CFL_LAMMAX_FLAT_BLK_NS_SRC.replace("sqrtf(u*u + v*v)", "fmaxf(fabsf(u), fabsf(v))").replace(
        "cfl_lammax_flat_blk_ns", "cfl_lammax_flat_blk_ns_linf")
    assert "fmaxf(fabsf(u), fabsf(v))" in lam_inf
    return {k2d.name: k2d.code, kres.name: kres.code, kres64.name: kres64.code,
            kfl.name: kfl.code, kfl_inf.name: kfl_inf.code,
            "cfl_lammax_flat_blk_ns": CS._CFL_LAMMAX_FLAT_BLK_NS_SRC, "cfl_lammax_flat_blk_ns_linf": lam_inf,
            "lammax_fp32_lean": S._CFL_LAMMAX_SRC_LEAN,
            # the flat loop's per-step forcings (compressed_solver.py:143-158, 268-283, 313-437, 1320-1328)
            "infiltrate_flat": CS._INFILTRATE_SRC, "drain_cap": CS._DRAIN_CAP_SRC,
            "ga_drain_flat": CS._GA_DRAIN_FLAT_SRC, "ga_flat": CS._GA_FLAT_SRC,
            "drain_tau_flat": CS._DRAIN_TAU_FLAT_SRC, "stage_clamp_flat": CS._STAGE_CLAMP_FLAT_SRC,
            "sponge_band": CS._SPONGE_BAND_SRC}


# C launch wrappers around the captured kernels (signatures of the reference text:
# rhs_cuda.py:900-914 + 2159-2162 for the 2-D fused step, solver.py:152-165 for lammax).
_WRAPPERS = r"""
#include <cuda_runtime.h>
extern "C" int ref_fstep2d(const float* q0, const float* q1, const float* q2, const float* b,
    float* qn0, float* qn1, float* qn2, int nxp, int nyp, float inv_dx, float inv_dy, float g,
    float h_min, const float* rain, int have_rain, const unsigned char* n_cls, const float* n_tab,
    const float* n_field, int use_tab, float* max_h, int have_max, int ngh, float dt, float vcap,
    int use_quadratic, const unsigned char* dummy_mask, const float* dummy_sigma, void* stream) {
    dim3 block(16, 16), grid((nxp + 15) / 16, (nyp + 15) / 16);
    fused_rhs_wb_srm_hllc_fstep2d_ns_fp32<<<grid, block, 0, (cudaStream_t)stream>>>(
        q0, q1, q2, dummy_sigma, b, qn0, qn1, qn2, nxp, nyp, inv_dx, inv_dy, g, h_min,
        dummy_mask, 0, qn0, qn1, qn2, rain, have_rain, n_field, n_cls, n_tab, use_tab,
        max_h, have_max, ngh, dt, vcap, use_quadratic);
    return (int)cudaGetLastError();
}
extern "C" int ref_rhs_f32(const float* q0, const float* q1, const float* q2, const float* b,
    float* r0, float* r1, float* r2, int nxp, int nyp, float inv_dx, float inv_dy, float g,
    float h_min, const unsigned char* mask, const float* dummy_sigma, void* stream) {
    dim3 block(16, 16), grid((nxp + 15) / 16, (nyp + 15) / 16);
    fused_rhs_wb_srm_hllc_2d_ns_fp32<<<grid, block, 0, (cudaStream_t)stream>>>(
        q0, q1, q2, dummy_sigma, b, r0, r1, r2, nxp, nyp, inv_dx, inv_dy, g, h_min, mask);
    return (int)cudaGetLastError();
}
extern "C" int ref_rhs_f64(const double* q0, const double* q1, const double* q2, const double* b,
    double* r0, double* r1, double* r2, int nxp, int nyp, double inv_dx, double inv_dy, double g,
    double h_min, const unsigned char* mask, const double* dummy_sigma, void* stream) {
    dim3 block(16, 16), grid((nxp + 15) / 16, (nyp + 15) / 16);
    fused_rhs_wb_srm_hllc_2d_ns_fp64<<<grid, block, 0, (cudaStream_t)stream>>>(
        q0, q1, q2, dummy_sigma, b, r0, r1, r2, nxp, nyp, inv_dx, inv_dy, g, h_min, mask);
    return (int)cudaGetLastError();
}
extern "C" int ref_forcing(int which, float* q0, float* q1, float* q2, const unsigned char* cls,
    const float* t0, const float* t1, const float* t2, float* F, const float* Fmax, const float* inv_tau,
    const unsigned char* act, const int* idx, const float* a0, const float* a1, int n, float dt, float h_min,
    void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = (n + 255) / 256;
    switch (which) {
    case 0: infiltrate_flat<<<grid, 256, 0, s>>>(q0, q1, q2, cls, t0, act, n, dt, h_min); break;
    case 1: sponge_band<<<grid, 256, 0, s>>>(idx, a0, a1, q0, q1, q2, n); break;
    case 2: ga_drain_flat<<<grid, 256, 0, s>>>(q0, q1, q2, cls, t0, t1, t2, F, Fmax, inv_tau, act, dt, n); break;
    case 3: ga_flat<<<grid, 256, 0, s>>>(q0, q1, q2, cls, t0, t1, t2, F, Fmax, act, dt, n); break;
    case 4: drain_tau_flat<<<grid, 256, 0, s>>>(q0, q1, q2, inv_tau, act, dt, n); break;
    case 5: stage_clamp_flat<<<grid, 256, 0, s>>>(idx, q0, q1, q2, a0, n); break;
    case 6: drain_cap<<<grid, 256, 0, s>>>(idx, q0, q1, q2, a0, n); break;
    default: return -1;
    }
    return (int)cudaGetLastError();
}
// the flat fused step + CFL (signature: rhs_cuda.py:900-914 with compressed_rhs.py:44-47,
// 687-694, 1100-1102; launched as CompressedStepper.rhs_fused, compressed_solver.py:880-905:
// 256 threads, region_mode 0, no sigma, inv_sig = a length-1 array of ones with stride 0)
extern "C" int ref_flat_fstep(int linf, const float* q0, const float* q1, const float* q2, const float* b,
    float* qn0, float* qn1, float* qn2, int N, float inv_dx, float g, float h_min, const short* nbr,
    const unsigned char* is_active, const float* rate_row, const int* lk, int have_rain, const float* ones1,
    const unsigned char* n_cls, const float* n_tab, float* max_h, int have_max, float dt, float vcap,
    int use_quadratic, unsigned int* cfl_bits, float h_min_cfl, float* dummy, void* stream) {
    const int grid = (N + 255) / 256;
    cudaStream_t s = (cudaStream_t)stream;
    if (linf)
        flat_srm_hllc_fstepcfl_chained_linf_ns_float<<<grid, 256, 0, s>>>(q0, q1, q2, dummy, b, dummy, dummy, dummy,
            N, 0, inv_dx, inv_dx, g, h_min, nbr, is_active, is_active, 0, qn0, qn1, qn2, rate_row, lk, have_rain,
            ones1, 0, n_cls, n_tab, max_h, have_max, dt, vcap, use_quadratic, cfl_bits, h_min_cfl, 0);
    else
        flat_srm_hllc_fstepcfl_chained_ns_float<<<grid, 256, 0, s>>>(q0, q1, q2, dummy, b, dummy, dummy, dummy,
            N, 0, inv_dx, inv_dx, g, h_min, nbr, is_active, is_active, 0, qn0, qn1, qn2, rate_row, lk, have_rain,
            ones1, 0, n_cls, n_tab, max_h, have_max, dt, vcap, use_quadratic, cfl_bits, h_min_cfl, 0);
    return (int)cudaGetLastError();
}
// the flat lammax (compressed_solver.py:200-244), launched as CompressedStepper.cfl_dt does
// (2048 blocks of 256, compressed_solver.py:735-739)
extern "C" int ref_flat_lammax(int linf, const float* q0, const float* q1, const float* q2,
    const unsigned char* act, int N, float g, float h_min, float h_min_cfl, unsigned int* out_bits,
    const float* dummy, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (linf) cfl_lammax_flat_blk_ns_linf<<<2048, 256, 0, s>>>(q0, q1, q2, dummy, act, N, g, h_min, h_min_cfl, out_bits);
    else cfl_lammax_flat_blk_ns<<<2048, 256, 0, s>>>(q0, q1, q2, dummy, act, N, g, h_min, h_min_cfl, out_bits);
    return (int)cudaGetLastError();
}
extern "C" int ref_lammax(const float* q0, const float* q1, const float* q2, int nx, int ny,
    int nyp, int ngh, float g, float h_cfl, unsigned int* out_bits, const unsigned char* ghost,
    void* stream) {
    const int N = nx * ny;
    int grid = (N + 255) / 256; if (grid > 2048) grid = 2048;
    lammax_fp32_lean<<<grid, 256, 0, (cudaStream_t)stream>>>(q0, q1, q2, N, nx, ny, nyp, ngh, g,
                                                               h_cfl, out_bits, ghost);
    return (int)cudaGetLastError();
}
"""


def reference_src():
    """The reference package's source directory: $GEOSWE_REFERENCE_SRC when set, else the
    checkout location of this build host. The GPU box has neither; nothing there needs it."""
    return Path(os.environ.get("GEOSWE_REFERENCE_SRC", "/root/reference/src"))


def build(ref_src=None):
    ref_src = Path(ref_src) if ref_src is not None else reference_src()
    if not Path(ref_src).exists():
        raise FileNotFoundError(f"reference tree {ref_src} not found (the recipe runs where it is)")
    srcs = capture(ref_src)
    OUT.mkdir(exist_ok=True)
    parts = []
    for name, code in srcs.items():
        parts.append(f"// ---- {name} (captured from the reference) ----\n")
        # each captured text defines its own macros (WETDRY_KEEP_H); keep them per kernel
        parts.append(code)
        parts.append("\n#undef WETDRY_KEEP_H\n#undef BSIZE\n#undef _RSTRIDE\n")
    cu = OUT / "ref_kernels.cu"
    cu.write_text("".join(parts) + _WRAPPERS)
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    for tag, extra in (("fma", []), ("strict", ["--fmad=false"])):
        out = OUT / f"libref_{tag}.so"
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", *extra,
                        "-Xcompiler", "-fPIC", "-shared", "-o", str(out), str(cu)], check=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference src directory (default: reference_src())")
    a = ap.parse_args()
    print(build(a.ref))
