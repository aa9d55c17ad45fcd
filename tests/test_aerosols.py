"""The climatological aerosol optics (setaer / aer_property, NAM iaer = 11) in the oracle, pinned to the
reference's own kernels: the float restatement reproduces the golden vectors of aer_init, clim_aerinit,
aer_update's month fill, setaer and aer_property bit for bit, and the packed climatology has the shape and
ranges the kernels assume.  The volcanic term (setaer's lavoflg branch) reproduces phys_rrtm_setaer_volc's
golden vectors in both level orders and with the one-broad-band LW factor.  The reference's surface-first
branches (ivflip 1) of setaer and aer_property mirror its top-first ones bit for bit, which is what lets the
restatement and the GPU path serve surface-first requests by reversing the layers."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from woof_nam_b200 import aerosols
from woof_nam_b200.columns import Columns, make_columns

GOLDEN = Path(__file__).resolve().parent / "golden" / "aer_golden.npz"
CASES = ("jan_nam", "jul_globe")
VOLC_CASES = {"top_first": (0, 0, 2026, 7), "surface_first": (1, 0, 1991, 6), "one_lw_band": (0, 1, 7, 12)}


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def golden_request(z, case):
    """(month, a Columns carrying plvl / plyr / tlyr / qlyr, the aerosol inputs)."""
    base = make_columns(z[f"{case}_in_plyr"].shape[1], 1)
    kw = {f: getattr(base, f) for f in Columns.FIELDS}
    for k in ("plvl", "plyr", "tlyr", "qlyr"):
        kw[k] = z[f"{case}_in_{k}"]
    ai = {k: z[f"{case}_in_{k}"] for k in ("rhly", "xlon", "xlat", "slmsk")}
    return int(z[f"{case}_in_month"][0]), Columns(**kw), ai


def test_packed_climatology():
    c = aerosols.climatology(3)
    assert c["month_idx"].shape == (37, 72, 5) and c["month_kprf"].shape == (37, 72)
    assert c["month_kprf"].min() >= 1 and c["month_kprf"].max() <= 7
    assert c["month_idx"].min() >= 0 and c["month_idx"].max() <= 10
    assert int(c["nwvns0"].sum()) == 57600 and c["iendwv"].shape == (61,)
    assert np.all(np.diff(c["iendwv"]) > 0)
    with pytest.raises(ValueError):
        aerosols.climatology(13)


@pytest.mark.parametrize("case", CASES)
def test_tables_bit_exact(gold, case):
    month, cols, ai = golden_request(gold, case)
    r = oracle.aerosols(aerosols.climatology(month), cols, ai, tables=True)
    for name, _ in oracle.AER_TAB_FIELDS:
        assert np.array_equal(r[name], gold[f"{case}_tab_{name}"]), name


@pytest.mark.parametrize("case", CASES)
def test_optics_bit_exact(gold, case):
    month, cols, ai = golden_request(gold, case)
    r = oracle.aerosols(aerosols.climatology(month), cols, ai)
    assert np.array_equal(r["faersw"], gold[f"{case}_faersw"])
    assert np.array_equal(r["faerlw"], gold[f"{case}_faerlw"])


@pytest.mark.parametrize("case", CASES)
def test_optics_ranges(gold, case):
    for k in ("faersw", "faerlw"):
        a = gold[f"{case}_{k}"]
        assert np.isfinite(a).all()
        assert (a[0] >= 0).all() and a[0].max() > 0            # optical depth
        assert ((a[1] >= 0) & (a[1] <= 1)).all()                # single-scattering albedo
        assert ((a[2] >= 0) & (a[2] <= 1)).all()                # asymmetry


def test_inputs_in_range():
    cols = make_columns(64, 5)
    for region in ("nam", "globe"):
        ai = aerosols.make_inputs(cols, 9, region)
        assert ai["rhly"].shape == (cols.nlay, cols.ncol) and 0 <= ai["rhly"].min() and ai["rhly"].max() <= 1
        assert np.abs(ai["xlat"]).max() <= np.pi / 2


@pytest.mark.parametrize("case", list(VOLC_CASES))
def test_volcanic_bit_exact(gold, case):
    ivflip, lw1bd, kyrsav, kmonsav = VOLC_CASES[case]
    pl = gold["jul_globe_in_plvl"]
    pl = pl if ivflip == 0 else np.ascontiguousarray(pl[::-1])
    r = oracle.setaer_volc(pl, gold["volc_in_xlat"], gold["volc_in_ivolae"], kyrsav, kmonsav,
                           gold["jul_globe_faersw"], gold["jul_globe_faerlw"], ivflip=ivflip, lw1bd=bool(lw1bd))
    assert np.array_equal(r["faersw"][0], gold[f"volc_{case}_extsw"])
    assert np.array_equal(r["faerlw"][0], gold[f"volc_{case}_extlw"])
    assert np.array_equal(r["faersw"][1:], gold["jul_globe_faersw"][1:])
    # the term lies between 5 mb and 250 mb at most, and adds to every column
    added = r["faerlw"][0] - gold["jul_globe_faerlw"][0]
    assert (added >= 0).all() and (added.sum(axis=(0, 1)) > 0).all()


def test_volcanic_switches(gold):
    pl, xl, iv = gold["jul_globe_in_plvl"], gold["volc_in_xlat"], gold["volc_in_ivolae"]
    sw, lw = gold["jul_globe_faersw"], gold["jul_globe_faerlw"]
    r = oracle.setaer_volc(pl, xl, iv, 3, 2, sw, lw, add_sw=False, add_lw=False)
    assert np.array_equal(r["faersw"], sw) and np.array_equal(r["faerlw"], lw)
    only_lw = oracle.setaer_volc(pl, xl, iv, 3, 2, sw, lw, add_sw=False)
    both = oracle.setaer_volc(pl, xl, iv, 3, 2, sw, lw)
    assert np.array_equal(only_lw["faersw"], sw) and np.array_equal(only_lw["faerlw"], both["faerlw"])
    # the year index is kyrsav mod 10 as Python takes it: -7 and 3 read the same year
    assert np.array_equal(oracle.setaer_volc(pl, xl, iv, -7, 2, sw, lw)["faersw"], both["faersw"])
    with pytest.raises(ValueError):
        oracle.setaer_volc(pl, xl, iv, 3, 13, sw, lw)


def test_surface_first_mirrors_top_first(gold):
    fl = lambda a: np.ascontiguousarray(np.asarray(a)[::-1])  # noqa: E731
    month, cols, ai = golden_request(gold, "jul_globe")
    for k in ("faersw", "faerlw"):   # the reference's own ivflip = 1 output is its ivflip = 0 output, reversed
        assert np.array_equal(gold[f"flip_{k}"], np.ascontiguousarray(gold[f"jul_globe_{k}"][:, :, ::-1]))
    r = oracle.aerosols(aerosols.climatology(month), oracle._Flip(cols, fl), dict(ai, rhly=fl(ai["rhly"])), ivflip=1)
    assert np.array_equal(r["faersw"], gold["flip_faersw"]) and np.array_equal(r["faerlw"], gold["flip_faerlw"])
