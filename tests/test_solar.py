"""The solar geometry of a radiation call (sol_update + coszmn) pinned to the reference's kernels: the
oracle's restatement and the library's host sol_update (rad_sol_update, no GPU needed) reproduce the golden
vectors bit for bit."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from woof_nam_b200 import solar

GOLDEN = Path(__file__).resolve().parent / "golden" / "solar_golden.npz"
STATE = ("sollag", "sindec", "cosdec", "anginc", "solcon")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_oracle_bit_exact(gold):
    for i in range(gold["date"].shape[0]):
        r = oracle.solar(gold["date"][i], float(gold["deltsw"][i]), float(gold["deltim"][i]), 1366.0,
                         gold["glon"][i], gold["glat"][i], float(gold["solhr"][i]), float(gold["dtswav"][i]), 48)
        assert np.array_equal(r["state"], gold["state"][i]) and r["nstp"] == gold["nstp"][i], i
        assert np.array_equal(r["coszen"], gold["coszen"][i]) and np.array_equal(r["coszdg"], gold["coszdg"][i]), i


def test_library_sol_update_bit_exact(gold):
    for i in range(gold["date"].shape[0]):
        s = solar.sol_update(gold["date"][i], float(gold["deltsw"][i]), float(gold["deltim"][i]), 1366.0)
        got = np.array([s[k] for k in STATE], np.float32)
        assert np.array_equal(got, gold["state"][i]) and s["nstp"] == gold["nstp"][i], i


def test_sol_update_ranges(gold):
    st = gold["state"]
    assert (np.abs(st[:, 1]) <= np.sin(np.deg2rad(23.5))).all()            # declination within the tropics
    assert np.allclose(st[:, 1] ** 2 + st[:, 2] ** 2, 1.0, atol=1e-6)
    assert ((st[:, 4] > 1366.0 * 0.96) & (st[:, 4] < 1366.0 * 1.04)).all()  # sun-earth distance +-1.7 %
    assert ((gold["coszen"] >= 0) & (gold["coszen"] <= 1)).all() and (gold["coszdg"] >= 0).all()
    # coszdg is the sum of the samples times dtswav / nrads (the reference's scaling, hours)
    assert (gold["coszdg"] <= gold["dtswav"][:, None] + 1e-6).all()


@pytest.mark.parametrize("bad", [dict(month=13), dict(hour=24), dict(deltim=0.0)])
def test_sol_update_rejects(bad):
    d = dict(year=2026, month=7, day=1, hour=12, minute=0, second=0, deltsw=1200.0, deltim=25.0)
    d.update(bad)
    with pytest.raises(ValueError):
        solar.sol_update((d["year"], d["month"], d["day"], d["hour"], d["minute"], d["second"]), d["deltsw"],
                         d["deltim"])
