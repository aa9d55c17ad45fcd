"""Generate rdtemp_golden.npz: the reference's own rdtemp_apply kernel (namgpu/kernels/drv_rdtemp.cu:
140-198), compiled for the host into oracle/_ref/libref_rrtm.so by oracle/build_ref.sh, on seeded inputs
(oracle.rdtemp.make_case: 24 x 16 columns, 10 levels) for three calendars (a non-leap March day, a leap-year
October day after 5,000 steps, 1 January 1999 at the start).

  c{n}_in_*       the inputs (arrays) of case n; c{n}_scal the scalars (ntsd, julday, julyr, ihrst,
                  leap_seen, and the eight 1-based limits), c{n}_dt the step
  c{n}_czen, c{n}_t  the reference kernel's outputs

Run from the repository root:  python tests/golden/make_rdtemp_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle, rdtemp  # noqa: E402

OUT = Path(__file__).resolve().parent / "rdtemp_golden.npz"
CASES = ((1, 73, 2025, 37), (2, 300, 2024, 5000), (3, 1, 1999, 0))
SCAL = ("ntsd", "julday", "julyr", "ihrst", "leap_seen", "its", "ite", "jts", "jte", "its_b1", "ite_b1", "jts_b1", "jte_b1")
ARR = ("glat", "glon", "czmean", "rswtt", "rlwtt", "t", "czen")


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    blob = {}
    for n, (seed, jd, yr, nt) in enumerate(CASES):
        p = rdtemp.make_case(24, 16, 10, seed, ntsd=nt, julday=jd, julyr=yr)
        r = rdtemp.reference_rdtemp(p)
        blob.update({f"c{n}_in_{k}": p[k] for k in ARR})
        blob[f"c{n}_scal"] = np.array([p[k] for k in SCAL], dtype=np.int32)
        blob[f"c{n}_dt"] = np.array([p["dt"]], dtype=np.float32)
        blob[f"c{n}_czen"], blob[f"c{n}_t"] = r["czen"], r["t"]
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
