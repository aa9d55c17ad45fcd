"""Generate the golden vectors in this directory from the reference's own radiation kernels.

The reference kernels (namgpu/kernels/phys_rrtm_*.cu) are compiled for the host by oracle/build_ref.sh
(oracle/_ref/libref_rrtm.so) and driven in the reference's call order by oracle/ref_driver.cpp, in the
reference's FP32 arithmetic.  That library exists only where the reference tree is mounted, so the
vectors are committed:

  rrtm_golden.npz
    in_*            the request (two seeded requests: 40 columns of the plain workload, 24 of the stress one)
    lw_*            LW outputs of the reference (float32)
    sw_*            SW outputs of the reference at full optical depth (float32; NaN where the reference's
                    float layer solver overflows -- kept to pin that behaviour)
    swq_*           SW outputs with every gas optical depth scaled by 1e-3 before the two-stream solver
                    (finite everywhere; pins the solver arithmetic)
    st_*            SW stage outputs (taug, taur, sfluxzen, cloud optics, laytrop) of the first 6 day columns
    mc{0,1,2}_*     McICA sub-column cloud words of the reference's LW / SW generators, overlap 0, 1, 2
    mcseed, mcs_*   the same for explicit seeds (overlap 1)

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from woof_nam_b200.columns import make_columns  # noqa: E402

OUT = Path(__file__).resolve().parent / "rrtm_golden.npz"
CASES = {"plain": (40, 1001, False), "stress": (24, 5005, True)}
NSTAGE = 6


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    blob = {}
    for case, (ncol, seed, stress) in CASES.items():
        cols = make_columns(ncol, seed, stress=stress)
        for f in cols.FIELDS:
            blob[f"{case}_in_{f}"] = np.asarray(getattr(cols, f), dtype=np.float32)
        blob[f"{case}_in_solcon"] = np.array([cols.solcon], dtype=np.float64)
        blob[f"{case}_in_diagnostic"] = np.array([int(cols.diagnostic_clouds)], dtype=np.int32)
        oracle.set_debug(1.0, which="ref")
        r = oracle.reference_solve(cols)
        for k in ("htlw", "topflw", "sfcflw"):
            blob[f"{case}_lw_{k}"] = r[k].astype(np.float32)
        for k in ("htsw", "topfsw", "sfcfsw", "fdncmp"):
            blob[f"{case}_sw_{k}"] = r[k].astype(np.float32)
        oracle.set_debug(1.0e-3, which="ref")
        r = oracle.reference_solve(cols)
        oracle.set_debug(1.0, which="ref")
        for k in ("htsw", "topfsw", "sfcfsw", "fdncmp"):
            blob[f"{case}_swq_{k}"] = r[k].astype(np.float32)
        st = oracle.sw_stages(cols, which="ref")
        for k, v in st.items():
            blob[f"{case}_st_{k}"] = v[:NSTAGE]
        for iovr in (0, 1, 2):
            m = oracle.mcica_masks(cols, which="ref", iovrlw=iovr, iovrsw=iovr)
            blob[f"{case}_mc{iovr}_lw"] = m["lw"]
            blob[f"{case}_mc{iovr}_sw"] = m["sw"]
        seeds = np.random.default_rng(seed).integers(-2**31, 2**31 - 1, size=(2, ncol)).astype(np.int32)
        m = oracle.mcica_masks(cols, which="ref", icseed=seeds)
        blob[f"{case}_mcseed"] = seeds
        blob[f"{case}_mcs_lw"] = m["lw"]
        blob[f"{case}_mcs_sw"] = m["sw"]
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
