"""The NAM route's other cloud overlaps in the oracle, pinned to the reference's own kernels: LW random
overlap (iovrlw = 0, rtrn) and the SW clear-sky view fraction with random / maximum overlap (iovrsw 0 / 2).
The float statements of the restatement reproduce the golden vectors bit for bit; the float64 restatement
stays within rounding of them."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import golden_columns, max_errors
from oracle import oracle
from woof_nam_b200.columns import make_columns

CASES = ("plain", "stress")
OVERLAP = Path(__file__).resolve().parent / "golden" / "overlap_golden.npz"


@pytest.fixture(scope="module")
def ovl():
    return np.load(OVERLAP)


def test_requests_are_60_layers(ovl):
    for case in CASES:
        assert golden_columns(ovl, case).nlay == 60


@pytest.mark.parametrize("case", CASES)
def test_rtrn_bit_exact(ovl, case):
    cols = golden_columns(ovl, case)
    r = oracle.solve(cols, precision="float", iovrlw=0)
    for k in ("htlw", "topflw", "sfcflw"):
        assert np.array_equal(r[k].astype(np.float32), ovl[f"{case}_rn_{k}"]), k


@pytest.mark.parametrize("case", CASES)
def test_rtrn_fp64_close_to_reference(ovl, case):
    cols = golden_columns(ovl, case)
    r = oracle.solve(cols, precision="double", iovrlw=0)
    ref = {k: ovl[f"{case}_rn_{k}"].astype(np.float64) for k in ("htlw", "topflw", "sfcflw")}
    e = max_errors(r, ref)
    assert e["htlw"] < 0.01 and e["topflw"] < 0.05 and e["sfcflw"] < 0.05, e


@pytest.mark.parametrize("case", CASES)
def test_random_overlap_is_a_different_transfer(ovl, case):
    """rtrn and rtrnmr agree on clear columns and differ where a column has more than one cloudy layer."""
    cols = golden_columns(ovl, case)
    rn = oracle.solve(cols, precision="float", iovrlw=0)
    mr = oracle.solve(cols, precision="float", iovrlw=1)
    assert not np.array_equal(rn["htlw"], mr["htlw"])
    clear = (cols.clouds[0] <= 1.0e-6).all(axis=0)
    if clear.any():
        assert np.array_equal(rn["htlw"][:, clear], mr["htlw"][:, clear])


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("iovr", [0, 2])
def test_sw_overlap_bit_exact(ovl, case, iovr):
    cols = golden_columns(ovl, case)
    oracle.set_debug(1.0e-3)
    try:
        r = oracle.solve(cols, precision="float", iovrsw=iovr)
    finally:
        oracle.set_debug(1.0)
    for k in ("htsw", "topfsw", "sfcfsw", "fdncmp"):
        assert np.array_equal(r[k].astype(np.float32), ovl[f"{case}_swq{iovr}_{k}"]), k


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("iovr", [0, 2])
def test_zcf_bit_exact(ovl, case, iovr):
    cols = golden_columns(ovl, case)
    z = oracle.sw_stages(cols, iovrsw=iovr)["zcf"]
    assert np.array_equal(z, ovl[f"{case}_zcf{iovr}"])


def test_zcf_ordering(ovl):
    """Clear-sky view fraction: random overlap <= maximum-random <= maximum (more overlap, more clear sky)."""
    cols = golden_columns(ovl, "plain")
    z = {i: oracle.sw_stages(cols, iovrsw=i)["zcf"][:, 0].astype(np.float64) for i in (0, 1, 2)}
    assert (z[0] <= z[1] + 1e-7).all() and (z[1] <= z[2] + 1e-7).all()


def test_reference_rtrn_refuses_61_layers():
    """The reference's rtrn holds at most 60 layers; its driver reports that instead of returning zeros."""
    if not oracle.REF_LIB.exists():
        pytest.skip("oracle/_ref is built only where the reference tree is present")
    with pytest.raises(RuntimeError):
        oracle.reference_solve(make_columns(8, 3), iovrlw=0)
