"""The NAM route's other cloud overlaps on the GPU (through the C-ABI) against the float64 oracle: LW random
overlap (iovrlw = 0, rtrn) in the two-kernel LW, the single-kernel LW and the FP64 kernel, and the SW
clear-sky view fraction with random / maximum overlap (iovrsw 0 / 2).  Tolerances as the max-random route:
0.05 W/m^2 and 0.01 K/day for the mixed precision."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_within, golden_columns
from oracle import oracle
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu


def _solver(**kw):
    from woof_nam_b200.solver import RadSolver
    return RadSolver(**kw)


@pytest.fixture(scope="module")
def plain():
    cols = make_columns(2048, 4242)
    return cols, oracle.solve(cols, precision="double", iovrlw=0, iovrsw=0)


@pytest.fixture(scope="module")
def stress():
    cols = make_columns(2048, 5151, stress=True)
    return cols, oracle.solve(cols, precision="double", iovrlw=0, iovrsw=2)


@pytest.mark.parametrize("lw_chunk", [0, 512, -1])
def test_mixed_random_overlap(plain, lw_chunk):
    cols, ref = plain
    out = _solver(precision="mixed", iovrlw=0, iovrsw=0, lw_chunk=lw_chunk).solve_host(cols)
    assert_within(out, ref, what=f"mixed, random overlap, lw_chunk {lw_chunk}")


def test_mixed_stress_random_overlap(stress):
    """The stress request's 0.1 hPa cloudy top layer sends its columns to the float64 LW fallback."""
    cols, ref = stress
    out = _solver(precision="mixed", diagnostic=True, iovrlw=0, iovrsw=2).solve_host(cols)
    assert_within(out, ref, what="mixed, random overlap, stress")


def test_fp64_random_overlap(plain, stress):
    """The FP64 kernel contracts multiply-adds, so a float64 optical depth on a lookup-table boundary can take
    the neighbouring entry of the oracle's: up to ~1e-3 K/day on single layers of 2,048 columns."""
    cols, ref = plain
    out = _solver(precision="fp64", iovrlw=0, iovrsw=0).solve_host(cols)
    assert_within(out, ref, flux_tol=2e-3, heat_tol=2e-3, what="fp64, random overlap")
    cols, ref = stress
    out = _solver(precision="fp64", diagnostic=True, iovrlw=0, iovrsw=2).solve_host(cols)
    assert_within(out, ref, flux_tol=2e-3, heat_tol=2e-3, what="fp64, random overlap, stress")


def test_iovrlw_2_is_rtrnmr(plain):
    """lwrad runs rtrnmr for every iovrlw > 0: iovrlw 2 gives the bits of iovrlw 1."""
    cols, _ = plain
    a = _solver(iovrlw=1).solve_host(cols)
    b = _solver(iovrlw=2).solve_host(cols)
    for k in ("htlw", "topflw", "sfcflw"):
        assert np.array_equal(a[k], b[k]), k


def test_golden_60_layers():
    """The 60-layer requests of the overlap golden vectors (the reference's rtrn limit): the FP64 kernel
    against the float64 oracle, and the oracle's float statements against the reference's outputs."""
    z = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "overlap_golden.npz")
    for case in ("plain", "stress"):
        cols = golden_columns(z, case)
        ref = oracle.solve(cols, precision="double", iovrlw=0)
        out = _solver(nlay=60, precision="fp64", diagnostic=cols.diagnostic_clouds, iovrlw=0).solve_host(cols)
        assert_within({k: out[k] for k in ("htlw", "topflw", "sfcflw")}, ref, flux_tol=2e-3, heat_tol=2e-3,
                      what=f"fp64 rtrn, 60 layers, {case}")
