"""Generate overlap_golden.npz, the golden vectors of the NAM route's other cloud overlaps, from the
reference's own kernels (oracle/_ref/libref_rrtm.so, built by oracle/build_ref.sh from the reference tree):

  LW  iovrlw = 0: lwrad's transfer is rtrn (random overlap, namgpu/kernels/phys_rrtm_lw_rtrn.cu) instead of
      rtrnmr.  The reference's rtrn holds at most 60 layers (phys_rrtm_lw_rtrn.py:60), so the requests here
      are the plain and stress workloads with the extra top radiation layer left out (60 layers).
  SW  iovrsw = 0 / 2: swrad's clear-sky view fraction zcf0 with random / maximum overlap
      (phys_rrtm_sw_swrad.cu:251-279).

Keys, per case (plain: 40 columns seed 1001, stress: 24 columns seed 5005):
    in_*            the 60-layer request
    rn_*            LW outputs with iovrlw = 0 (float32)
    swq{0,2}_*      SW outputs with iovrsw 0 / 2, gas optical depths x 1e-3 before the two-stream solver
                    (finite everywhere; full-depth SW overflows to NaN in the reference's float solver)
    zcf{0,2}        zcf0, zcf1 of the day columns, iovrsw 0 / 2

Run from the repository root:  python tests/golden/make_overlap_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from woof_nam_b200.columns import Columns, make_columns  # noqa: E402

OUT = Path(__file__).resolve().parent / "overlap_golden.npz"
CASES = {"plain": (40, 1001, False), "stress": (24, 5005, True)}


def without_top_layer(c: Columns) -> Columns:
    """The request with its first (top) radiation layer and interface removed."""
    kw = {}
    for f in c.FIELDS:
        a = getattr(c, f)
        if f in ("plyr", "tlyr", "qlyr", "olyr", "plvl", "tlvl"):
            a = a[1:]
        elif f in ("gasvmr", "clouds"):
            a = a[:, 1:]
        kw[f] = np.ascontiguousarray(a, dtype=np.float32)
    return Columns(**kw, solcon=c.solcon, diagnostic_clouds=c.diagnostic_clouds)


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    blob = {}
    for case, (ncol, seed, stress) in CASES.items():
        cols = without_top_layer(make_columns(ncol, seed, stress=stress))
        for f in cols.FIELDS:
            blob[f"{case}_in_{f}"] = getattr(cols, f)
        blob[f"{case}_in_solcon"] = np.array([cols.solcon], dtype=np.float64)
        blob[f"{case}_in_diagnostic"] = np.array([int(cols.diagnostic_clouds)], dtype=np.int32)
        oracle.set_debug(1.0, which="ref")
        r = oracle.reference_solve(cols, iovrlw=0)
        for k in ("htlw", "topflw", "sfcflw"):
            blob[f"{case}_rn_{k}"] = r[k].astype(np.float32)
        oracle.set_debug(1.0e-3, which="ref")
        for iovr in (0, 2):
            r = oracle.reference_solve(cols, iovrsw=iovr)
            for k in ("htsw", "topfsw", "sfcfsw", "fdncmp"):
                blob[f"{case}_swq{iovr}_{k}"] = r[k].astype(np.float32)
        oracle.set_debug(1.0, which="ref")
        for iovr in (0, 2):
            blob[f"{case}_zcf{iovr}"] = oracle.sw_stages(cols, which="ref", iovrsw=iovr)["zcf"]
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
