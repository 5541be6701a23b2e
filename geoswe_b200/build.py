"""Build libgsw.so (the sm_100a kernels and their C ABI) in the package directory.

    python -m geoswe_b200.build            # compile if a source is newer than the .so
    python -m geoswe_b200.build --force    # always recompile

The library is compiled with ``--fmad=false``: every multiply and add of the step is
rounded separately, in the reference's operand order, so the C oracle reproduces the
kernels' values exactly. The one exception is gsw_fast.cu, the opt-in fast-arithmetic
compilation of the binary32 step kernels (FMA contraction, flush-to-zero). Only nvcc
is needed; no GPU is touched.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libgsw.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
# The fast-arithmetic compilation of the binary32 step kernels (gsw_fast.cu): FMA
# contraction and flush-to-zero; its square root and division are the approximate
# instructions named in gsw_core.cuh.
FAST_SOURCES = {"gsw_fast.cu"}
FAST_FLAGS = [f for f in NVCC_FLAGS if f != "--fmad=false"] + ["--fmad=true", "-ftz=true"]


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def source_hash(names=None) -> str:
    """First 16 hex digits of the SHA-256 over the library's sources and headers (name
    and content, in name order), or over the files called `names` only (the sources a
    kernel is compiled from): names the build a profile was captured on."""
    import hashlib
    h = hashlib.sha256()
    files = sources() + headers()
    if names is not None:
        files = [p for p in files if p.name in set(names)]
    for p in sorted(files, key=lambda q: q.name):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()[:16]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources() + headers())


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    if not force and not needs_build():
        return LIB
    objs = []
    build_dir = PKG / "_build"
    build_dir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        flags = FAST_FLAGS if src.name in FAST_SOURCES else NVCC_FLAGS
        cmd = [nvcc, *ARCH, *flags, *extra, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = [nvcc, "-x", "c++", "-Wno-deprecated-gpu-targets", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-fvisibility=hidden", *extra, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print register/spill usage")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    out = build(force=a.force or a.ptxas_info, verbose=a.verbose, extra=extra)
    print(out)


if __name__ == "__main__":
    sys.exit(main())
