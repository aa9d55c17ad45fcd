"""Build libradb200.so (the CUDA kernels and the C ABI) in-tree for sm_100a with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
LIB = PKG / "libradb200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def sources():
    return sorted(SRC.glob("*.cu")) + sorted(SRC.glob("*.cuh")) + sorted(SRC.glob("*.h")) + \
        [PKG.parent / "include" / "radb200.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile csrc/rad_capi.cu (which includes the solve's kernel headers) and csrc/rad_front.cu (grrad's front
    end, its own translation unit) and link them into libradb200.so."""
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in sources()):
        return LIB
    base = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
    if verbose:
        base.append("-Xptxas=-v")
    # The solve: float division / square root to within 2 ulp and float denormals flushed -- the mixed kernels'
    # arithmetic is arranged so that neither changes results beyond the float rounding they already carry; the
    # plain FP64 kernels and every float64 statement are unaffected.
    solve = ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
    # The front end: every statement rounded as written (IEEE division and square root, denormals kept, no
    # multiply-add contraction), as the single-precision routines it restates.
    front = ["-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-fmad=false"]
    with tempfile.TemporaryDirectory() as tmp:
        objs, procs = [], []
        for src, flags in (("rad_capi.cu", solve), ("rad_front.cu", front)):   # the two units side by side
            obj = str(Path(tmp) / (src + ".o"))
            procs.append(subprocess.Popen([*base, *flags, "-c", "-o", obj, str(SRC / src)]))
            objs.append(obj)
        for p, src in zip(procs, ("rad_capi.cu", "rad_front.cu")):
            if p.wait() != 0:
                raise subprocess.CalledProcessError(p.returncode, f"nvcc {src}")
        subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *objs], check=True)
    return LIB

if __name__ == "__main__":
    build(force=True, verbose=True)
    print(LIB)
