"""grrad's front end in the oracle, pinned to the reference's kernels: the restatement (oracle/rrtm_front.hpp)
reproduces the golden vectors of phys_rrtm_dayparts_*, phys_rrtm_getgases, phys_rrtm_getozn, phys_rrtm_setalb,
phys_rrtm_setemis, phys_rrtm_progcld2_column, grrad's condensate (grrad_clouds_clw) and its IALB = 2 surface
albedo (grrad_clouds_albedo, whose built-in tables the packed woof_nam_b200/data/payne_albedo.npz reproduces) bit
for bit in every flag branch, and the DAYPARTS run table
and gethml's deck indices have the structure the consumers rely on (grrad_nmmb.f:640-653)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

GOLDEN = Path(__file__).resolve().parent / "golden" / "front_golden.npz"
GAS_CASES = {f"co2_{f}_flip{v}": (f, v) for f in (0, 1, 2) for v in (0, 1)}
OZN = dict(k1oz=3, k2oz=4, facoz=0.37, blte=-85.0, dlte=10.0)
EMIS_CASES = {f"alb{a}_lw{lw}": (a, lw) for a in (0, 1) for lw in (0, 1)}
CLD_CASES = ("nam", "sashal_random", "flip", "flip_sashal", "thompson")
CLW_CASES = ((2, 1), (2, 3))
PAYNE = Path(__file__).resolve().parents[1] / "woof_nam_b200" / "data" / "payne_albedo.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def _in(z, prefix):
    n = len(prefix) + 4
    return {k[n:]: z[k] for k in z.files if k.startswith(prefix + "_in_")}


def _flip(a):
    return np.ascontiguousarray(np.asarray(a)[::-1])


def test_dayparts(gold):
    d = _in(gold, "dp")
    im = int(gold["dp_in_xlon"].size // gold["dp_ndayparts"].size)
    r = oracle.dayparts(d["xlon"], d["sinlat"], d["coslat"], im, float(d["scal"][0]), float(d["scal"][1]),
                        int(d["nrads"]), d["sol"])
    for k in r:
        assert np.array_equal(r[k], gold[f"dp_{k}"]), k
    # each row's runs tile the row, alternate day and night, and agree with the point flags
    day = (r["coszen"] >= np.float32(1e-4)).reshape(-1, im)
    for j, nr in enumerate(r["ndayparts"]):
        s, ln, dd = (r[k][j * im:j * im + nr] for k in ("dp_start", "dp_len", "dp_day"))
        assert s[0] == 1 and (s[1:] == s[:-1] + ln[:-1]).all() and ln.sum() == im
        assert (dd[1:] != dd[:-1]).all()
        for a, b, f in zip(s, ln, dd):
            assert (day[j, a - 1:a - 1 + b] == f).all()
        assert (r["dp_start"][j * im + nr:(j + 1) * im] == -1).all()       # slots past the runs untouched


@pytest.mark.parametrize("case", list(GAS_CASES))
def test_getgases(gold, case):
    f, v = GAS_CASES[case]
    pl = gold["lay_in_plvl"] if v == 0 else _flip(gold["lay_in_plvl"])
    g = oracle.getgases(pl, gold["sfc_in_glon"], gold["sfc_in_glat"], float(gold["tab_in_co2_glb"]),
                        gold["tab_in_gco2cyc"], gold["tab_in_co2vmr_sav"], f, 7, v)
    assert np.array_equal(g, gold[f"gas_{case}_gasvmr"])


@pytest.mark.parametrize("flip", [0, 1])
def test_getozn(gold, flip):
    pk = gold["lay_in_prslk1"] if flip == 0 else _flip(gold["lay_in_prslk1"])
    o = oracle.getozn(pk, gold["sfc_in_glat"], gold["tab_in_o3r"], gold["tab_in_pkstr"], OZN["k1oz"], OZN["k2oz"],
                      OZN["facoz"], OZN["blte"], OZN["dlte"], flip)
    assert np.array_equal(o, gold[f"ozn_flip{flip}_o3mmr"], equal_nan=True)
    assert np.isnan(o).any()      # the extra top layer lies above the climatology's first level: left alone


@pytest.mark.parametrize("ialbflg", [0, 1, 2])
def test_setalb(gold, ialbflg):
    assert np.array_equal(oracle.setalb(_in(gold, "sfc"), ialbflg), gold[f"alb_{ialbflg}_sfcalb"])


@pytest.mark.parametrize("case", list(EMIS_CASES))
def test_setemis(gold, case):
    a, lw = EMIS_CASES[case]
    e = oracle.setemis(_in(gold, "sfc"), gold["tab_in_idxems"], a, lw)
    assert np.array_equal(e, gold[f"ems_{case}_sfcemis"])


@pytest.mark.parametrize("case", CLD_CASES)
def test_progcld2(gold, case):
    c = gold[f"cld_{case}_cfg"]
    cfg = dict(zip(oracle.CLD_CFG, c.tolist()))
    cld = _in(gold, "cld")
    if cfg["ivflip"]:
        cld = {k: (v if k == "xlat" else _flip(v)) for k, v in cld.items()}
    r = oracle.progcld2(cld, cfg)
    for k in r:
        assert np.array_equal(r[k], gold[f"cld_{case}_{k}"]), k
    nlay = cld["plyr"].shape[0]
    assert ((r["mtop"] >= 1) & (r["mtop"] <= nlay) & (r["mbot"] >= 1) & (r["mbot"] <= nlay)).all()
    cl = r["clds"]
    assert ((cl >= 0) & (cl <= 1)).all() and (cl[3] >= cl[:3].max(0) - 1e-6).all()   # total >= each deck


@pytest.mark.parametrize("ntcw,ncld", CLW_CASES)
def test_grrad_clw(gold, ntcw, ncld):
    r = oracle.grrad_clw(gold["clw_in_tracer"], ntcw, ncld)
    assert np.array_equal(r, gold[f"clw_{ntcw}_{ncld}_clw"])
    assert (r == 0).any() and (r > 0).any()
    with pytest.raises(ValueError):
        oracle.grrad_clw(gold["clw_in_tracer"], 3, 3)


def test_payne_albedo(gold):
    tables = dict(np.load(PAYNE))
    assert tables["albd"].shape == (20, 21) and tables["za"][0] == 90.0 and tables["za"][-1] == 0.0
    r = oracle.payne_albedo(gold["payne_in_salbedo"], gold["payne_in_sm"], gold["payne_in_coszen"], tables)
    for k in oracle.PAYNE_OUT:
        assert np.array_equal(r[k], gold[f"payne_{k}"]), k
    changed = r["sfcalbedo"] != gold["payne_in_salbedo"]
    assert changed.any() and (~changed).any()
    assert not changed[(gold["payne_in_sm"] <= 0.5) | (gold["payne_in_coszen"] <= 0)].any()
