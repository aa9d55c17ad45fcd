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

the surface-first orientation (ivflip 1) of the "jul_globe" request, its layers flipped, through the reference's
ivflip = 1 branches of setaer's prep and aer_property:
    flip_faersw, flip_faerlw   [3][14|16][nlay][ncol], layers surface first

and the volcanic term (setaer's lavoflg branch, orc_setaer_volc: phys_rrtm_setaer_prep then
phys_rrtm_setaer_volc) added to the "jul_globe" optics, per case of VOLC_CASES (ivflip, lw1bd, kyrsav,
kmonsav), on a seeded ivolae table and latitudes across the seven zone bands and their edges:
    volc_in_ivolae, volc_in_xlat, volc_<case>_extsw [14][nlay][ncol], volc_<case>_extlw [16][nlay][ncol]
(the term changes the extinction, component 0, only)

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
VOLC_CASES = {"top_first": (0, 0, 2026, 7), "surface_first": (1, 0, 1991, 6), "one_lw_band": (0, 1, 7, 12)}


def volc_inputs(ncol: int, seed: int = 303):
    """ivolae int32 [10][4][12] and latitudes (radians) in every zone band and on the band edges."""
    r = np.random.default_rng(seed)
    ivolae = r.integers(0, 500, (10, 4, 12)).astype(np.int32)
    deg = np.array([89.0, 72.0, 46.0, 45.5, 44.0, 30.0, 1.0, 0.25, -1.0, -20.0, -44.0, -45.0, -46.0, -70.0, -80.5,
                    -90.0][:ncol], np.float32)
    return ivolae, np.radians(deg).astype(np.float32)


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
    fl = lambda a: np.ascontiguousarray(np.asarray(a)[::-1])  # noqa: E731
    month, ncol, seed, region = CASES["jul_globe"]
    cols = make_columns(ncol, seed)
    ai = aerosols.make_inputs(cols, seed, region)
    r = oracle.aerosols(aerosols.climatology(month), oracle._Flip(cols, fl), dict(ai, rhly=fl(ai["rhly"])),
                        which="ref", ivflip=1)
    blob["flip_faersw"], blob["flip_faerlw"] = r["faersw"], r["faerlw"]
    ivolae, xlat = volc_inputs(16)
    blob["volc_in_ivolae"], blob["volc_in_xlat"] = ivolae, xlat
    plvl = blob["jul_globe_in_plvl"]
    for case, (ivflip, lw1bd, kyrsav, kmonsav) in VOLC_CASES.items():
        pl = plvl if ivflip == 0 else np.ascontiguousarray(plvl[::-1])
        v = oracle.setaer_volc(pl, xlat, ivolae, kyrsav, kmonsav, blob["jul_globe_faersw"], blob["jul_globe_faerlw"],
                               ivflip=ivflip, lw1bd=bool(lw1bd), which="ref")
        for k in ("faersw", "faerlw"):
            assert np.array_equal(v[k][1:], blob[f"jul_globe_{k}"][1:])
        blob[f"volc_{case}_extsw"], blob[f"volc_{case}_extlw"] = v["faersw"][0], v["faerlw"][0]
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
