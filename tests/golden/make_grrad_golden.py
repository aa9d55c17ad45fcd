"""Generate grrad_golden.npz, the golden vectors of grrad's radiation-layer set-up, from the reference's own
kernels rrtm_grrad_setup and phys_rrtm_grrad_gases (oracle/_ref/libref_rrtm.so, built by oracle/build_ref.sh)
on the model state of two seeded requests (columns.model_state of make_columns: 48 plain columns, 32 of the
precision-stress request with its 0.1 hPa top layer).

Keys, per case: in_pint, in_pmid, in_prslk, in_t, in_q, in_tsfc (the model state), then plvl, plyr, tlyr,
tlvl, qlyr, rhly, qstl, prslk1, tvly, tsfg (oracle.GRRAD_FIELDS).

Run from the repository root:  python tests/golden/make_grrad_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from woof_nam_b200.columns import make_columns, model_state  # noqa: E402

OUT = Path(__file__).resolve().parent / "grrad_golden.npz"
CASES = {"plain": (48, 1001, False), "stress": (32, 5005, True)}


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    blob = {}
    for case, (n, seed, stress) in CASES.items():
        m = model_state(make_columns(n, seed, stress=stress))
        for k, v in m.items():
            blob[f"{case}_in_{k}"] = v
        for k, v in oracle.grrad_setup(m, which="ref").items():
            blob[f"{case}_{k}"] = v
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
