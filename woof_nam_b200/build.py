"""Build libradb200.so (the CUDA kernels and the C ABI) in-tree for sm_100a with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess
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
    """Compile csrc/rad_capi.cu (which includes the kernel headers) into libradb200.so."""
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in sources()):
        return LIB
    # float division / square root to within 2 ulp and float denormals flushed: the mixed kernels'
    # arithmetic is arranged so that neither changes results beyond the float rounding they already carry;
    # the plain FP64 kernels and every float64 statement are unaffected.
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-prec-div=false", "-prec-sqrt=false", "-ftz=true",
           "-Xcompiler", "-fPIC", "-shared",
           "-o", str(LIB), str(SRC / "rad_capi.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
    print(LIB)
