"""Generate solar_golden.npz, the golden vectors of the radiation call's solar geometry, from the reference's
own kernels sol_update_nmmb and phys_rrtm_coszmn (oracle/_ref/libref_rrtm.so, built by oracle/build_ref.sh):
48 seeded forecast times (1990-2039, SW intervals of 10 min to 3 h, model steps of 12.5 to 30 s), each with
the sun's state and the daytime / whole-interval mean zenith cosines of 64 seeded columns (48 samples).

Keys: date [48, 6], deltsw, deltim [48], state [48, 5] (sollag, sindec, cosdec, anginc, solcon), nstp [48],
glon, glat [48, 64] (radians), solhr, dtswav [48], coszen, coszdg [48, 64].

Run from the repository root:  python tests/golden/make_solar_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent / "solar_golden.npz"
NCASE, NCOL, NRADS, SOLC0 = 48, 64, 48, 1366.0


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    rng = np.random.default_rng(2026)
    b = {k: [] for k in ("date", "deltsw", "deltim", "state", "nstp", "glon", "glat", "solhr", "dtswav", "coszen",
                         "coszdg")}
    for _ in range(NCASE):
        date = [int(rng.integers(1990, 2040)), int(rng.integers(1, 13)), int(rng.integers(1, 29)),
                int(rng.integers(0, 24)), int(rng.integers(0, 60)), int(rng.integers(0, 60))]
        dsw, dt = float(rng.choice([600.0, 1200.0, 3600.0, 10800.0])), float(rng.choice([12.5, 25.0, 30.0]))
        lon = rng.uniform(-np.pi, 2 * np.pi, NCOL).astype(np.float32)
        lat = rng.uniform(-1.55, 1.55, NCOL).astype(np.float32)
        solhr = np.float32(date[3] + date[4] / 60.0)
        dtsw = np.float32(dsw / 3600.0)
        r = oracle.solar(date, dsw, dt, SOLC0, lon, lat, float(solhr), float(dtsw), NRADS, which="ref")
        for k, v in (("date", date), ("deltsw", dsw), ("deltim", dt), ("state", r["state"]), ("nstp", r["nstp"]),
                     ("glon", lon), ("glat", lat), ("solhr", solhr), ("dtswav", dtsw), ("coszen", r["coszen"]),
                     ("coszdg", r["coszdg"])):
            b[k].append(v)
    blob = {k: np.array(v) for k, v in b.items()}
    blob["date"] = blob["date"].astype(np.int32)
    blob["nstp"] = blob["nstp"].astype(np.int32)
    for k in ("deltsw", "deltim", "solhr", "dtswav"):
        blob[k] = blob[k].astype(np.float32)
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
