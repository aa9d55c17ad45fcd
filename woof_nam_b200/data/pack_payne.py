"""Pack the surface-albedo tables of grrad's IALB = 2 block (the DATA statements TRN, ZA, DZA and ALBD of
grrad_nmmb.f, as the reference's namgpu/kernels/phys_rrtm_grrad_clouds.cu:186-250 holds them) into
``payne_albedo.npz`` next to this script: trn [21] (transmissivity steps), za [20] (zenith angles, degrees),
dza [19] (their spacing) and albd [20][21] (albedo by zenith-angle row and transmissivity column, the Fortran
ALBD(21, 20) read column-major).  The packed file is what the library, the oracle and the tests load; nothing
at run time reads the reference tree.

Usage:  python woof_nam_b200/data/pack_payne.py REFERENCE_ROOT
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "payne_albedo.npz"
SIZES = {"c_TRN": 21, "c_ZA": 20, "c_DZA": 19, "c_ALBD": 420}


def read_tables(source: str) -> dict:
    out = {}
    for name, n in SIZES.items():
        m = re.search(name + r"\[\d+\]\s*=\s*\{([^}]*)\}", source)
        if m is None:
            raise SystemExit(f"{name} not found")
        vals = [float(v.rstrip("fF")) for v in re.findall(r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?[fF]?", m.group(1))]
        if len(vals) != n:
            raise SystemExit(f"{name}: {len(vals)} values, expected {n}")
        out[name] = np.array(vals, np.float32)
    return out


def main():
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    src = (Path(sys.argv[1]) / "namgpu" / "kernels" / "phys_rrtm_grrad_clouds.cu").read_text()
    t = read_tables(src)
    np.savez_compressed(OUT, trn=t["c_TRN"], za=t["c_ZA"], dza=t["c_DZA"], albd=t["c_ALBD"].reshape(20, 21))
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
