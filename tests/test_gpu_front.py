"""grrad's front end on the GPU through the C-ABI (rad_dayparts, rad_getgases, rad_getozn, rad_setalb,
rad_setemis, rad_progcld2) against the golden vectors of the reference's kernels and against the oracle at the
parent domain's size (954 x 835 points, 65,536 cloud columns).

The front-end kernels round every statement as written (IEEE division and square root, no contraction), so
getgases, getozn, setemis and the albedo of ialbflg 2 agree bit for bit, and so does progcld2's NAM
configuration apart from the effective radii.  Where CUDA's cosf / powf / expf enter, values agree to within
their last-bit differences: a relative 4e-6 for the direct sea albedo and the effective radii, an absolute
5e-7 for the zenith cosines (a sum of cosines that may cancel to near zero), and a relative 1e-4 for the cloud
fraction of the humidity forms (1 - expf(-v), whose relative rounding grows as it nears the 1e-3 cloud limit).
The integer outputs (the DAYPARTS run table, gethml's deck layers) agree bit for bit; at the parent domain's
size a day flag may differ where the oracle's zenith cosine lies within that rounding of the 1e-4 day limit,
and the GPU's run table must then be exactly the run-length code of its own flags."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from woof_nam_b200.columns import cloud_state, front_tables, make_columns, model_state, surface_state

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "front_golden.npz"
GAS_CASES = {f"co2_{f}_flip{v}": (f, v) for f in (0, 1, 2) for v in (0, 1)}
OZN = dict(k1oz=3, k2oz=4, facoz=0.37, blte=-85.0, dlte=10.0)
EMIS_CASES = {f"alb{a}_lw{lw}": (a, lw) for a in (0, 1) for lw in (0, 1)}
CLD_CASES = ("nam", "sashal_random", "flip", "flip_sashal", "thompson")
RTOL = 4e-6


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def solver():
    from woof_nam_b200.solver import RadSolver
    return RadSolver()


def _cuda(a, dtype=None):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype), device="cuda")


def _np(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _in(z, prefix):
    n = len(prefix) + 4
    return {k[n:]: z[k] for k in z.files if k.startswith(prefix + "_in_")}


def _flip(a):
    return np.ascontiguousarray(np.asarray(a)[::-1])


def _close(g, r, what, rtol=RTOL, atol=0.0):
    assert g.shape == r.shape, what
    if g.dtype.kind in "iu":
        assert np.array_equal(g, r), what
        return
    fin = np.isfinite(r)
    assert np.array_equal(np.isfinite(g), fin), what
    d = np.abs(g[fin].astype(np.float64) - r[fin])
    bad = d > atol + rtol * np.abs(r[fin]).astype(np.float64)
    assert not bad.any(), (what, float(d.max()), int(bad.sum()))


def _runs(day, im):
    """Run-length code of per-point day flags, row by row (the DAYPARTS table), slots past the runs -1."""
    n = day.size
    st, ln, dd, nr = np.full(n, -1, np.int32), np.full(n, -1, np.int32), np.full(n, -1, np.int32), []
    for j in range(n // im):
        f = day[j * im:(j + 1) * im].astype(np.int32)
        s = np.flatnonzero(np.r_[True, f[1:] != f[:-1]])
        e = np.r_[s[1:], im]
        k = s.size
        st[j * im:j * im + k], ln[j * im:j * im + k], dd[j * im:j * im + k] = s + 1, e - s, f[s]
        nr.append(k)
    return {"dp_start": st, "dp_len": ln, "dp_day": dd, "ndayparts": np.array(nr, np.int32)}


def _sun(sol):
    from woof_nam_b200 import _lib
    s = _lib.RadSolarState(float(sol[0]), float(sol[1]), float(sol[2]), 0.0, 0.0, 1)
    return {"_state": s}


def _dayparts(solver, xlon, sinlat, coslat, im, solhr, dtswav, nrads, sol):
    from woof_nam_b200 import front
    out = {}
    n = xlon.size
    import torch
    for k in ("dp_start", "dp_len", "dp_day"):
        out[k] = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    out["ndayparts"] = torch.zeros(n // im, dtype=torch.int32, device="cuda")
    out["coszen"] = torch.empty(n, dtype=torch.float32, device="cuda")
    out["coszdg"] = torch.empty(n, dtype=torch.float32, device="cuda")
    r = front.dayparts(solver, _cuda(xlon), _cuda(sinlat), _cuda(coslat), solhr, dtswav, nrads, _sun(sol), im, out=out)
    return {k: _np(v) for k, v in r.items()}


def test_dayparts_golden(gold, solver):
    d = _in(gold, "dp")
    im = int(d["xlon"].size // gold["dp_ndayparts"].size)
    r = _dayparts(solver, d["xlon"], d["sinlat"], d["coslat"], im, float(d["scal"][0]), float(d["scal"][1]),
                  int(d["nrads"]), d["sol"])
    for k in r:
        _close(r[k], gold[f"dp_{k}"], f"dayparts {k}", rtol=0.0, atol=5e-7)


@pytest.mark.parametrize("im,jm,nrads", [(954, 835, 8), (24576, 3, 2), (1, 5, 3), (257, 2, 1)])
def test_dayparts_against_oracle(solver, im, jm, nrads):
    """The parent domain; the longest row the kernel takes; one-point rows; a row one point past a tile."""
    r = np.random.default_rng(im + jm)
    lon = np.sort(r.uniform(-np.pi, np.pi, (jm, im)), axis=1).astype(np.float32).ravel()
    lat = r.uniform(-1.55, 1.55, jm * im).astype(np.float32)
    if im == 24576:       # flip the day flag every few points along the row
        lon = r.uniform(-np.pi, np.pi, jm * im).astype(np.float32)
    sol = np.array([0.02, -0.3, 0.954], np.float32)
    args = (lon, np.sin(lat).astype(np.float32), np.cos(lat).astype(np.float32), im, 7.75, 1.0 / 3.0, nrads, sol)
    g = _dayparts(solver, *args)
    o = oracle.dayparts(*args)
    for k in ("coszen", "coszdg"):
        _close(g[k], o[k], f"dayparts {im}x{jm} {k}", rtol=0.0, atol=5e-7)
    lim = np.float32(1e-4)
    gd, od = g["coszen"] >= lim, o["coszen"] >= lim
    flips = np.flatnonzero(gd != od)
    assert (np.abs(o["coszen"][flips].astype(np.float64) - 1e-4) < 5e-7).all(), "a day flag differs away from the limit"
    own = _runs(gd, im)
    for k in own:
        assert np.array_equal(g[k], own[k]), f"dayparts {im}x{jm} {k}: not the run-length code of the GPU's flags"
        if flips.size == 0:
            assert np.array_equal(g[k], o[k]), f"dayparts {im}x{jm} {k}"


@pytest.mark.parametrize("case", list(GAS_CASES))
def test_getgases_golden(gold, solver, case):
    from woof_nam_b200 import front
    f, v = GAS_CASES[case]
    pl = gold["lay_in_plvl"] if v == 0 else _flip(gold["lay_in_plvl"])
    g = front.getgases(solver, _cuda(pl), _cuda(gold["sfc_in_glon"]), _cuda(gold["sfc_in_glat"]),
                       co2_glb=_cuda(np.atleast_1d(gold["tab_in_co2_glb"])), gco2cyc=_cuda(gold["tab_in_gco2cyc"]),
                       co2vmr_sav=_cuda(gold["tab_in_co2vmr_sav"]), ico2flg=f, kmonsav=7, ivflip=v)
    assert np.array_equal(_np(g), gold[f"gas_{case}_gasvmr"])


@pytest.mark.parametrize("flip", [0, 1])
def test_getozn_golden(gold, solver, flip):
    import torch
    from woof_nam_b200 import front
    pk = gold["lay_in_prslk1"] if flip == 0 else _flip(gold["lay_in_prslk1"])
    init = torch.full(pk.shape, float("nan"), dtype=torch.float32, device="cuda")
    o = front.getozn(solver, _cuda(pk), _cuda(gold["sfc_in_glat"]), init, o3r=_cuda(gold["tab_in_o3r"]),
                     pkstr=_cuda(gold["tab_in_pkstr"]), ivflip=flip, **OZN)
    assert np.array_equal(_np(o), gold[f"ozn_flip{flip}_o3mmr"], equal_nan=True)


@pytest.mark.parametrize("ialbflg", [0, 1, 2])
def test_setalb_golden(gold, solver, ialbflg):
    from woof_nam_b200 import front
    sfc = {k: _cuda(v) for k, v in _in(gold, "sfc").items()}
    a = _np(front.setalb(solver, sfc, ialbflg))
    _close(a, gold[f"alb_{ialbflg}_sfcalb"], f"setalb {ialbflg}")
    if ialbflg == 2:
        assert np.array_equal(a, gold["alb_2_sfcalb"])


@pytest.mark.parametrize("case", list(EMIS_CASES))
def test_setemis_golden(gold, solver, case):
    from woof_nam_b200 import front
    a, lw = EMIS_CASES[case]
    sfc = {k: _cuda(v) for k, v in _in(gold, "sfc").items()}
    e = front.setemis(solver, sfc, _cuda(gold["tab_in_idxems"], np.int32), a, lw)
    assert np.array_equal(_np(e), gold[f"ems_{case}_sfcemis"])


def test_setemis_map_cells(solver):
    """The O(1) cell lookup finds the Fortran's first matching cell on and next to every cell boundary and
    centre, at the poles and the date line, and falls back to cell 1 where none matches."""
    from woof_nam_b200 import front
    deg = np.float32(np.pi / 180.0)
    lon = np.concatenate([np.arange(-180.0, 180.5, 0.25), [-180.0001, 179.9999, 359.9, 720.0, np.nan]])
    lat = np.concatenate([np.arange(-90.0, 90.01, 0.125), [90.4999, 90.5, 90.5001, -90.6, np.inf]])
    n = max(lon.size, lat.size)
    lon = (np.resize(lon, n) * deg).astype(np.float32)
    lat = (np.resize(lat[::-1], n) * deg).astype(np.float32)
    sfc = {"glon": lon, "glat": lat, "sm": np.zeros(n, np.float32), "sice": np.zeros(n, np.float32),
           "si": np.zeros(n, np.float32), "sncovr": np.zeros(n, np.float32), "z0": np.full(n, 0.1, np.float32),
           "stdh": np.zeros(n, np.float32), "tskin": np.full(n, 280.0, np.float32)}
    idx = (np.arange(180 * 360).reshape(180, 360) % 5 + 2).astype(np.int32)
    ref = oracle.setemis(sfc, idx, 0, 1)
    g = _np(front.setemis(solver, {k: _cuda(v) for k, v in sfc.items()}, _cuda(idx, np.int32), 0, 1))
    assert np.array_equal(g, ref)


@pytest.mark.parametrize("case", CLD_CASES)
def test_progcld2_golden(gold, solver, case):
    from woof_nam_b200 import front
    c = gold[f"cld_{case}_cfg"].tolist()
    cfg = dict(zip(oracle.CLD_CFG, c))
    cld = _in(gold, "cld")
    if cfg["ivflip"]:
        cld = {k: (v if k == "xlat" else _flip(v)) for k, v in cld.items()}
    r = front.progcld2(solver, {k: _cuda(v) for k, v in cld.items()}, **cfg)
    humid = cfg["cld_fraction"] == 0 and (cfg["ivflip"] != 0 or cfg["lsashal"] != 0)   # 1 - expf(-v) fraction
    for k in ("clouds", "clds", "mtop", "mbot"):
        _close(_np(r[k]), gold[f"cld_{case}_{k}"], f"progcld2 {case} {k}", rtol=1e-4 if humid else RTOL)
    if case == "nam":     # no transcendental in the NAM fraction: fractions and paths bit for bit
        cl = _np(r["clouds"])
        for q in (0, 1, 3, 5, 6):
            assert np.array_equal(cl[q], gold["cld_nam_clouds"][q]), q


def test_front_end_at_scale(solver):
    """65,536 columns: the layers of grrad's set-up, then progcld2, getgases, getozn, setalb and setemis on the
    GPU, each against the oracle on the same inputs."""
    from woof_nam_b200 import front
    n = 65536
    cols = make_columns(n, 77)
    lay = oracle.grrad_setup(model_state(cols))
    tab, sfc = front_tables(5), surface_state(n, 6)
    cld = cloud_state(lay, 8)
    cfg = dict(ivflip=0, llyr=2, iovr=1, lcrick=0, lcnorm=0, lnoprec=0, lsashal=0, cld_fraction=0)
    g = front.progcld2(solver, {k: _cuda(v) for k, v in cld.items()}, **cfg)
    o = oracle.progcld2(cld, cfg)
    for k in o:
        _close(_np(g[k]), o[k], f"progcld2 {k}")
    gas = front.getgases(solver, _cuda(lay["plvl"]), _cuda(sfc["glon"]), _cuda(sfc["glat"]),
                         co2_glb=_cuda(np.atleast_1d(tab["co2_glb"])), gco2cyc=_cuda(tab["gco2cyc"]),
                         co2vmr_sav=_cuda(tab["co2vmr_sav"]), ico2flg=2, kmonsav=11, ivflip=0)
    assert np.array_equal(_np(gas), oracle.getgases(lay["plvl"], sfc["glon"], sfc["glat"], tab["co2_glb"],
                                                    tab["gco2cyc"], tab["co2vmr_sav"], 2, 11, 0))
    oz = front.getozn(solver, _cuda(lay["prslk1"]), _cuda(sfc["glat"]), o3r=_cuda(tab["o3r"]),
                      pkstr=_cuda(tab["pkstr"]), k1oz=12, k2oz=1, facoz=0.8, blte=-85.0, dlte=10.0)
    ref = oracle.getozn(lay["prslk1"], sfc["glat"], tab["o3r"], tab["pkstr"], 12, 1, 0.8, -85.0, 10.0, 0,
                        init=np.zeros_like(lay["prslk1"]))
    assert np.array_equal(_np(oz), ref)
    sd = {k: _cuda(v) for k, v in sfc.items()}
    for a in (0, 1, 2):
        _close(_np(front.setalb(solver, sd, a)), oracle.setalb(sfc, a), f"setalb {a}")
    assert np.array_equal(_np(front.setemis(solver, sd, _cuda(tab["idxems"], np.int32), 1, 1)),
                          oracle.setemis(sfc, tab["idxems"], 1, 1))


def test_invalid_arguments(solver):
    from woof_nam_b200 import front
    from woof_nam_b200._lib import RAD_E_INVALID, RadError
    z = _cuda(np.zeros((3, 4), np.float32))
    v = _cuda(np.zeros(4, np.float32))
    tab = dict(co2_glb=_cuda(np.ones(1, np.float32)), gco2cyc=_cuda(np.zeros(12, np.float32)),
               co2vmr_sav=_cuda(np.zeros((12, 12, 24), np.float32)))
    with pytest.raises(RadError) as e:
        front.getgases(solver, z, v, v, ico2flg=3, kmonsav=1, ivflip=0, **tab)
    assert e.value.code == RAD_E_INVALID
    with pytest.raises(RadError):
        front.getgases(solver, z, v, v, ico2flg=1, kmonsav=13, ivflip=0, **tab)
    with pytest.raises(RadError):
        front.getozn(solver, z, v, o3r=_cuda(np.zeros((12, 70, 18), np.float32)), pkstr=_cuda(np.zeros(70, np.float32)),
                     k1oz=1, k2oz=2, facoz=0.5, blte=-85.0, dlte=10.0)
    with pytest.raises(RadError):
        front.getozn(solver, z, v, o3r=_cuda(np.zeros((12, 17, 18), np.float32)), pkstr=_cuda(np.zeros(17, np.float32)),
                     k1oz=0, k2oz=2, facoz=0.5, blte=-85.0, dlte=10.0)
    cld = {k: z for k in ("plyr", "tlyr", "tvly", "qlyr", "qstl", "rhly", "clw", "f_ice", "f_rain", "cldfk1")}
    cld.update(plvl=_cuda(np.zeros((4, 4), np.float32)), xlat=v)
    with pytest.raises(RadError):
        front.progcld2(solver, cld, ivflip=0, llyr=4, iovr=1)             # llyr outside 1..nlay
    with pytest.raises(ValueError):
        front.dayparts(solver, v, v, v, 0.0, 1.0, 1, _sun([0, 0, 1]), 3)   # 4 points are not rows of 3


@pytest.mark.parametrize("ntcw,ncld", [(2, 1), (2, 3)])
def test_grrad_clw_golden(gold, solver, ntcw, ncld):
    """grrad's condensate: float sums in tracer order, bit for bit."""
    import torch
    from woof_nam_b200 import front
    clw = front.grrad_clw(solver, _cuda(gold["clw_in_tracer"]), ntcw, ncld)
    torch.cuda.synchronize()
    assert np.array_equal(clw.cpu().numpy(), gold[f"clw_{ntcw}_{ncld}_clw"])


def test_payne_albedo_golden(gold, solver):
    """grrad's IALB = 2 albedo with the packed tables against the reference kernel's built-in ones: CUDA's acosf
    against the host's moves the zenith angle by its last bits, and the table interpolation is continuous across
    rows, so the albedo agrees to 2e-6; the points the block leaves alone, and the copied fields, bit for bit."""
    import torch
    from woof_nam_b200 import front
    out = front.payne_albedo(solver, _cuda(gold["payne_in_salbedo"]), _cuda(gold["payne_in_sm"]),
                             _cuda(gold["payne_in_coszen"]))
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items()}
    for k in ("smx", "czmean", "facsf", "facwf"):
        assert np.array_equal(got[k], gold[f"payne_{k}"]), k
    keep = gold["payne_sfcalbedo"] == gold["payne_in_salbedo"]
    for k in ("sfcalbedo", "alvsf", "alnsf", "alvwf", "alnwf"):
        assert np.array_equal(got[k][keep], gold[f"payne_{k}"][keep]), k
        assert np.abs(got[k] - gold[f"payne_{k}"]).max() <= 2e-6, k
