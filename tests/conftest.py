"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built libradb200.so; the rest run on
the CPU (oracle against the golden vectors, the C-ABI surface, host-side logic, gloo ranks)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "rrtm_golden.npz"

# Tolerances of the mixed-precision path against the float64 oracle (fluxes W/m^2, heating K/day).
FLUX_TOL = 0.05
HEAT_TOL = 0.01
FLUX_KEYS = ("topflw", "sfcflw", "topfsw", "sfcfsw", "fdncmp")
HEAT_KEYS = ("htlw", "htsw")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libradb200.so")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def golden_columns(z, case: str):
    from woof_nam_b200.columns import Columns
    kw = {f: z[f"{case}_in_{f}"] for f in Columns.FIELDS}
    return Columns(**kw, solcon=float(z[f"{case}_in_solcon"][0]),
                   diagnostic_clouds=bool(z[f"{case}_in_diagnostic"][0]))


def max_errors(out: dict, ref: dict) -> dict:
    """Largest absolute error per output: heating rates in K/day, fluxes in W/m^2.  A value that is not
    finite where the reference is finite (or the other way round) counts as an infinite error."""
    e = {}
    for k in HEAT_KEYS + FLUX_KEYS:
        if k in out and k in ref:
            o = np.asarray(out[k], np.float64)
            r = np.asarray(ref[k], np.float64)
            if o.size == 0:
                e[k] = 0.0
                continue
            if not np.array_equal(np.isfinite(o), np.isfinite(r)):
                e[k] = float("inf")
                continue
            m = np.isfinite(r)
            d = np.abs(o[m] - r[m])
            e[k] = float(d.max() if d.size else 0.0) * (86400.0 if k in HEAT_KEYS else 1.0)
    return e


def assert_within(out: dict, ref: dict, flux_tol: float = FLUX_TOL, heat_tol: float = HEAT_TOL, what: str = ""):
    e = max_errors(out, ref)
    bad = {k: v for k, v in e.items() if v > (heat_tol if k in HEAT_KEYS else flux_tol)}
    assert not bad, f"{what} errors above tolerance (heat {heat_tol} K/day, flux {flux_tol} W/m^2): {bad}; all: {e}"
    return e
