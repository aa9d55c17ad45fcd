"""Generate aer_golden.npz, the golden vectors of the aerosol optics, from the reference's own kernels
(oracle/_ref/libref_rrtm.so, built by oracle/build_ref.sh from the reference tree): aer_init, clim_aerinit,
aer_update's month fill, setaer and aer_property, driven as the reference's wrappers drive them
(oracle/ref_driver.cpp orc_aerosols) on the packed climatology (woof_nam_b200/data/aer_tables.npz).

Keys, per case ("jan_nam": January, 16 columns over the NAM domain; "jul_globe": July, 16 columns anywhere):
    in_*        the request (plvl, plyr, tlyr, qlyr of make_columns; rhly, xlon, xlat, slmsk of
                aerosols.make_inputs) and the month
    faersw      [3][14][nlay][ncol] optical depth, single-scattering albedo, asymmetry (float32)
    faerlw      [3][16][nlay][ncol]
    tab_*       the derived tables (oracle.AER_TAB_FIELDS)

Run from the repository root:  python tests/golden/make_aer_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from woof_nam_b200 import aerosols  # noqa: E402
from woof_nam_b200.columns import make_columns  # noqa: E402

OUT = Path(__file__).resolve().parent / "aer_golden.npz"
CASES = {"jan_nam": (1, 16, 301, "nam"), "jul_globe": (7, 16, 302, "globe")}


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    blob = {}
    for case, (month, ncol, seed, region) in CASES.items():
        cols = make_columns(ncol, seed)
        ai = aerosols.make_inputs(cols, seed, region)
        r = oracle.aerosols(aerosols.climatology(month), cols, ai, which="ref", tables=True)
        for k in ("plvl", "plyr", "tlyr", "qlyr"):
            blob[f"{case}_in_{k}"] = np.asarray(getattr(cols, k), np.float32)
        for k, v in ai.items():
            blob[f"{case}_in_{k}"] = v
        blob[f"{case}_in_month"] = np.array([month], np.int32)
        blob[f"{case}_faersw"] = r["faersw"]
        blob[f"{case}_faerlw"] = r["faerlw"]
        for name, _ in oracle.AER_TAB_FIELDS:
            blob[f"{case}_tab_{name}"] = r[name]
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
