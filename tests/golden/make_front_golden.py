"""Generate front_golden.npz, the golden vectors of grrad's front end, from the reference's own kernels
(oracle/_ref/libref_rrtm.so, built by oracle/build_ref.sh): phys_rrtm_dayparts_cosz / _scatter / _len (with the
run-start scan), phys_rrtm_getgases, phys_rrtm_getozn, phys_rrtm_setalb, phys_rrtm_setemis and
phys_rrtm_progcld2_column, grrad_clouds_clw and grrad_clouds_albedo (the IALB = 2 block, with the reference's own
tables), on seeded synthetic inputs (columns.front_tables, surface_state, cloud_state; the
radiation layers of make_columns through grrad's set-up).  Every flag branch of each routine is a case.

Keys: <unit>_in_<name> for the inputs, <unit>_<case>_<output> for the outputs, and the case parameters as
<unit>_<case>_cfg where a case has some.

Run from the repository root:  python tests/golden/make_front_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from woof_nam_b200.columns import (cloud_state, front_tables, make_columns, model_state,  # noqa: E402
                                   surface_state)

OUT = Path(__file__).resolve().parent / "front_golden.npz"
N = 160                       # columns of the column routines
DP_IM, DP_JM = 131, 7         # DAYPARTS rows
GAS_CASES = {f"co2_{f}_flip{v}": (f, v) for f in (0, 1, 2) for v in (0, 1)}
OZN = dict(k1oz=3, k2oz=4, facoz=0.37, blte=-85.0, dlte=10.0)
EMIS_CASES = {f"alb{a}_lw{lw}": (a, lw) for a in (0, 1) for lw in (0, 1)}
CLW_CASES = ((2, 1), (2, 3))     # ntcw (1-based), ncld
CLD_CASES = {   # ivflip, llyr, iovr, lcrick, lcnorm, lnoprec, lsashal, cld_fraction
    "nam": (0, 2, 1, 0, 0, 0, 0, 0),
    "sashal_random": (0, 5, 0, 1, 1, 0, 1, 0),
    "flip": (1, 3, 1, 1, 0, 1, 0, 0),
    "flip_sashal": (1, 2, 0, 0, 1, 1, 1, 0),
    "thompson": (0, 2, 1, 0, 1, 1, 0, 1),
}


def dayparts_inputs(seed: int = 41) -> dict:
    """Points along rows whose longitudes cross the terminator, with latitudes into the polar day and night."""
    r = np.random.default_rng(seed)
    lon = np.linspace(-np.pi, np.pi, DP_IM, dtype=np.float32)[None, :] + r.uniform(-0.05, 0.05, (DP_JM, DP_IM))
    lat = np.linspace(-1.5, 1.5, DP_JM)[:, None] + r.uniform(-0.02, 0.02, (DP_JM, DP_IM))
    lat = lat.astype(np.float32)
    return {"xlon": lon.astype(np.float32).ravel(), "sinlat": np.sin(lat).ravel().astype(np.float32),
            "coslat": np.cos(lat).ravel().astype(np.float32), "sol": np.array([0.01, 0.35, 0.937], np.float32),
            "scal": np.array([13.25, 1.0 / 3.0], np.float32), "nrads": np.int32(4)}


def flip(a):
    return np.ascontiguousarray(np.asarray(a)[::-1])


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh <reference tree> first")
    blob = {}
    # DAYPARTS
    d = dayparts_inputs()
    for k, v in d.items():
        blob[f"dp_in_{k}"] = v
    res = oracle.dayparts(d["xlon"], d["sinlat"], d["coslat"], DP_IM, float(d["scal"][0]), float(d["scal"][1]),
                          int(d["nrads"]), d["sol"], which="ref")
    for k, v in res.items():
        blob[f"dp_{k}"] = v
    # the column routines' inputs
    cols = make_columns(N, 2024)
    lay = oracle.grrad_setup(model_state(cols), which="ref")
    sfc = surface_state(N, 2025)
    tab = front_tables(2026)
    for k in ("plvl", "prslk1"):
        blob[f"lay_in_{k}"] = lay[k]
    for k, v in sfc.items():
        blob[f"sfc_in_{k}"] = v
    for k, v in tab.items():
        blob[f"tab_in_{k}"] = np.asarray(v)
    # getgases
    for case, (f, v) in GAS_CASES.items():
        pl = lay["plvl"] if v == 0 else flip(lay["plvl"])
        blob[f"gas_{case}_gasvmr"] = oracle.getgases(pl, sfc["glon"], sfc["glat"], tab["co2_glb"], tab["gco2cyc"],
                                                     tab["co2vmr_sav"], f, 7, v, which="ref")
    # getozn (the routine leaves some levels alone: they start as NaN)
    for v in (0, 1):
        pk = lay["prslk1"] if v == 0 else flip(lay["prslk1"])
        blob[f"ozn_flip{v}_o3mmr"] = oracle.getozn(pk, sfc["glat"], tab["o3r"], tab["pkstr"], OZN["k1oz"],
                                                   OZN["k2oz"], OZN["facoz"], OZN["blte"], OZN["dlte"], v, which="ref")
    # setalb, setemis
    for a in (0, 1, 2):
        blob[f"alb_{a}_sfcalb"] = oracle.setalb(sfc, a, which="ref")
    for case, (a, lw) in EMIS_CASES.items():
        blob[f"ems_{case}_sfcemis"] = oracle.setemis(sfc, tab["idxems"], a, lw, which="ref")
    # progcld2
    cld = cloud_state(lay, 2027)
    for k, v in cld.items():
        blob[f"cld_in_{k}"] = v
    for case, c in CLD_CASES.items():
        cfg = dict(zip(oracle.CLD_CFG, c))
        inp = cld if c[0] == 0 else {k: (v if k == "xlat" else flip(v)) for k, v in cld.items()}
        for k, v in oracle.progcld2(inp, cfg, which="ref").items():
            blob[f"cld_{case}_{k}"] = v
        blob[f"cld_{case}_cfg"] = np.array(c, np.int32)
    # grrad's condensate (grrad_clouds_clw): four tracers, sums of one and of three from the second
    r = np.random.default_rng(44)
    tracer = (r.random((4, 61, N)) * r.choice([0.0, 1e-13, 1e-6, 1e-3], (4, 61, N))).astype(np.float32)
    blob["clw_in_tracer"] = tracer
    for ntcw, ncld in CLW_CASES:
        blob[f"clw_{ntcw}_{ncld}_clw"] = oracle.grrad_clw(tracer, ntcw, ncld, which="ref")
    # grrad's IALB = 2 albedo (grrad_clouds_albedo, the reference's built-in tables), zenith angles across every
    # row of the table including the overhead sun
    deg = np.concatenate([np.linspace(0.0, 95.0, N - 4), [74.0, 50.0, 89.99, 0.0]])
    pa = {"salbedo": r.uniform(0.05, 0.8, N).astype(np.float32),
          "sm": r.choice(np.array([0.0, 0.4, 0.6, 1.0], np.float32), N),
          "coszen": np.cos(np.radians(deg)).astype(np.float32)}
    for k, v in pa.items():
        blob[f"payne_in_{k}"] = v
    tables = dict(np.load(ROOT / "woof_nam_b200" / "data" / "payne_albedo.npz"))
    for k, v in oracle.payne_albedo(pa["salbedo"], pa["sm"], pa["coszen"], tables, which="ref").items():
        blob[f"payne_{k}"] = v
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
