"""Known answers of the McICA sub-column generators (the reference checks the same properties,
tools/check-phys-rrtm-lw-mcica-subcol.py:233-256 and tools/check-phys-rrtm-sw-mcica-subcol.py:177-210),
and the McICA route of the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from woof_nam_b200.columns import make_columns


def bits(words: np.ndarray, ngpt: int) -> np.ndarray:
    """[nword][nlay][ncol] uint32 -> bool [ngpt][nlay][ncol]."""
    nw, nlay, ncol = words.shape
    b = np.unpackbits(words.astype("<u4").view(np.uint8).reshape(nw, nlay, ncol, 4), axis=-1, bitorder="little")
    return b.transpose(0, 3, 1, 2).reshape(nw * 32, nlay, ncol)[:ngpt].astype(bool)


def with_cloud(cols, cf: float):
    cols.clouds[0][:] = np.float32(cf)
    return cols


@pytest.mark.parametrize("iovr", [0, 1, 2])
def test_clear_and_overcast(iovr):
    cols = with_cloud(make_columns(32, 5), 0.0)
    m = oracle.mcica_masks(cols, iovrlw=iovr, iovrsw=iovr)
    # a draw of exactly 1.0 (tempered words in [-128, -1] as int32) passes 1 - 0 >= 1: rare, not impossible
    assert bits(m["lw"], 140).mean() < 1e-4 and bits(m["sw"], 112).mean() < 1e-4
    cols = with_cloud(make_columns(32, 5), 1.0)
    m = oracle.mcica_masks(cols, iovrlw=iovr, iovrsw=iovr)
    assert bits(m["lw"], 140).all() and bits(m["sw"], 112).all()
    assert not (m["lw"][4] >> 12).any()   # words carry no bits past g-point 139


@pytest.mark.parametrize("iovr", [0, 1, 2])
def test_mean_follows_cloud_fraction(iovr):
    cols = with_cloud(make_columns(400, 9), 0.3)
    m = oracle.mcica_masks(cols, iovrlw=iovr, iovrsw=iovr)
    for key, ng in (("lw", 140), ("sw", 112)):
        assert abs(bits(m[key], ng).mean() - 0.3) < 0.01, key


def test_maximum_overlap_nests():
    """Maximum overlap: a sub-column cloudy in a layer is cloudy in every layer of larger cloud fraction."""
    cols = make_columns(64, 13)
    m = oracle.mcica_masks(cols, iovrlw=2, iovrsw=2)
    b = bits(m["sw"], 112)
    cf = cols.clouds[0][::-1]             # surface first
    for c in range(cols.ncol):
        order = np.argsort(cf[:, c], kind="stable")
        for i, j in zip(order[:-1], order[1:]):
            if cf[i, c] < cf[j, c] and cf[i, c] >= 1e-12:
                assert not (b[:, i, c] & ~b[:, j, c]).any()


def test_mcica_route_finite_and_close_to_nam():
    """The McICA route samples the same clouds: column fluxes stay finite and near the NAM route's."""
    cols = make_columns(256, 21)
    a = oracle.solve(cols, precision="double")
    b = oracle.solve(cols, precision="double", route=1)
    for k in ("htlw", "htsw", "topflw", "sfcflw", "topfsw", "sfcfsw"):
        assert np.isfinite(b[k]).all(), k
    assert abs(b["topflw"][0].mean() - a["topflw"][0].mean()) < 5.0
    assert np.array_equal(a["topflw"][1], b["topflw"][1])   # clear-sky TOA LW does not see the clouds
