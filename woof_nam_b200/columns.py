"""Seeded synthetic RRTM column states in the reference's radiation-driver layout.

The reference's real-case inputs are fetched from NOAA at run time and are not available offline, so
every workload here is generated.  The layout is exactly what the reference's ``lwrad``/``swrad``
entries read (``physics/rrtm/phys_rrtm_lw_lwrad.py:36-46``, ``physics/rrtm/phys_rrtm_sw_swrad.py:34-43``):
``[field, level, column]`` float32, level 0 = model top (ivflip = 0), with the reference's extra
radiation top layer (``kernels/phys_rrtm_grrad_setup.cu:185-200``: plvl(top) = prsmin = 1e-6 mb,
plyr(top) = plvl(1)/2, tlyr/qlyr copied from the layer below), so 60 model layers give nlay = 61,
nlp1 = 62.  Level temperatures follow the reference's log-pressure interpolation
(``kernels/phys_rrtm_grrad_gases.cu:20-31``): tlvl(top) = tlyr(top), tlvl(sfc) = skin temperature.

Generators (one rule each, as the workload definitions state them):

* pressure: surface U(950, 1030) hPa, model top 2 hPa, 60 hybrid sigma-pressure layers (pure pressure
  above 300 hPa, terrain-following below);
* temperature: 288 K + N(0, 5) at the surface, 6.5 K/km lapse (T = Ts (p/ps)^(R*gamma/g)) down to an
  isothermal 217 K at and above the 200 hPa tropopause;
* humidity: RH ~ U(0.1, 0.95) per layer, q from the Bolton (1980) saturation vapour pressure over
  water; above the tropopause q is capped at 3 ppm (mass) so the stratosphere stays dry;
* ozone: a climatological profile peaking at 8 ppmv at 10 hPa (Gaussian in ln p, width 1.2), floor
  0.03 ppmv, passed as a mass mixing ratio;
* gases: CO2 420 ppmv; N2O, CH4, O2, CO and the CFCs at the reference defaults
  (``kernels/phys_rrtm_getgases.cu:56-65``);
* clouds: fraction clip((RH - 0.8)/0.2, 0, 1); per column a liquid water path lognormal(median 50 g/m2,
  sigma 1) and an ice water path lognormal(median 20 g/m2, sigma 1), spread over the cloudy layers in
  proportion to cloud fraction x liquid share (ice share), liquid share clip((T - 253 K)/20 K, 0, 1), so
  the in-cloud layer paths sum (fraction-weighted) to the column paths; r_e = 10 um liquid, 50 um ice;
  no rain or snow;
* surface: albedo U(0.06, 0.8) in all four components, emissivity U(0.95, 1.0), skin temperature =
  lowest-layer temperature + N(0, 3);
* sun: cos(zenith) U(-1, 1), night where it is <= 0; solar constant 1368.22 W/m2;
* aerosol: none (the workloads give none).

The precision-stress workload switches to the diagnostic cloud-optics input form (cloud optical depth,
single-scattering albedo and asymmetry given directly: ``kernels/phys_rrtm_sw_cldprop.cu`` iswcliq = 0,
``kernels/phys_rrtm_lw_cldprop.cu`` ilwcliq = 0), with optical depth up to 500, SSA in [1-1e-7, 1],
cos(zenith) in [0.01, 0.05] and a 0.1 hPa thick model top layer.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

NLEV_MODEL = 60
NF_VGAS = 10
NF_CLDS = 9
AMD = 28.9644
AMO3 = 47.9982
PRSMIN = 1.0e-6
SOLCON = 1368.22
# gasvmr slots (reference getgases order): co2, n2o, ch4, o2, co, cfc11, cfc12, cfc22, ccl4, cfc113
GAS_DEFAULTS = (420.0e-6, 0.31e-6, 1.50e-6, 0.209, 1.50e-8, 3.520e-10, 6.358e-10, 1.500e-10, 1.397e-10,
                8.2000e-11)

# Column counts of the named workloads (12 km parent grid and the 3 km nests).
PARENT = (954, 835)
NESTS = ((333, 333), (600, 450), (180, 180))


@dataclass
class Columns:
    """One request's column state, [field, level, column] float32, level 0 = model top."""
    plyr: np.ndarray
    plvl: np.ndarray
    tlyr: np.ndarray
    tlvl: np.ndarray
    qlyr: np.ndarray
    olyr: np.ndarray
    gasvmr: np.ndarray
    clouds: np.ndarray
    sfcemis: np.ndarray
    tsfg: np.ndarray
    sfcalb: np.ndarray
    coszen: np.ndarray
    solcon: float = SOLCON
    diagnostic_clouds: bool = False

    @property
    def ncol(self) -> int:
        return int(self.plyr.shape[1])

    @property
    def nlay(self) -> int:
        return int(self.plyr.shape[0])

    FIELDS = ("plyr", "plvl", "tlyr", "tlvl", "qlyr", "olyr", "gasvmr", "clouds", "sfcemis", "tsfg",
              "sfcalb", "coszen")

    def arrays(self) -> dict:
        return {f: getattr(self, f) for f in self.FIELDS}

    def slice(self, c0: int, c1: int) -> "Columns":
        kw = {f: np.ascontiguousarray(getattr(self, f)[..., c0:c1]) for f in self.FIELDS}
        return Columns(**kw, solcon=self.solcon, diagnostic_clouds=self.diagnostic_clouds)

    def nbytes(self) -> int:
        return sum(getattr(self, f).nbytes for f in self.FIELDS)


def _esat_hpa(t):
    """Bolton (1980) saturation vapour pressure over water, hPa."""
    tc = t - 273.15
    return 6.112 * np.exp(17.67 * tc / (tc + 243.5))


def _interfaces(ps, ptop, top_thick=None):
    """Hybrid sigma-pressure interface pressures [61, ncol], hPa, top first."""
    n = NLEV_MODEL
    s = (np.arange(n + 1, dtype=np.float64) / n) ** 1.4          # finer spacing near the top
    pt2 = 300.0
    s_t = ((pt2 - ptop) / (1000.0 - ptop)) ** 1.0
    a = np.where(s < s_t, ptop + (pt2 - ptop) * s / s_t, pt2)
    b = np.where(s < s_t, 0.0, (s - s_t) / (1.0 - s_t))
    p = a[:, None] + b[:, None] * (ps[None, :] - pt2)
    if top_thick is not None:                                    # force the model top layer thickness
        p[1] = ptop + top_thick
    return p


def make_columns(ncol: int, seed: int, stress: bool = False) -> Columns:
    """Generate ``ncol`` columns with ``numpy.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    ptop = 2.0
    ps = rng.uniform(950.0, 1030.0, ncol)
    pi = _interfaces(ps, ptop, top_thick=0.1 if stress else None)           # [61, ncol]
    pl = 0.5 * (pi[:-1] + pi[1:])                                            # [60, ncol]
    ts = 288.0 + rng.normal(0.0, 5.0, ncol)
    kappa = 287.04 * 0.0065 / 9.80665
    t = ts[None, :] * (pl / ps[None, :]) ** kappa
    t = np.where(pl < 200.0, 217.0, np.maximum(t, 217.0))
    rh = rng.uniform(0.1, 0.95, (NLEV_MODEL, ncol))
    es = np.minimum(_esat_hpa(t), 0.5 * pl)
    qs = 0.622 * es / (pl - 0.378 * es)
    q = rh * qs
    q = np.where(pl < 200.0, np.minimum(q, 3.0e-6), q)
    q = np.maximum(q, 1.0e-7)
    o3v = 8.0e-6 * np.exp(-np.log(pl / 10.0) ** 2 / (2.0 * 1.2 ** 2))
    o3v = np.maximum(o3v, 0.03e-6)
    o3 = o3v * AMO3 / AMD

    # cloud fraction from RH; paths only where cloudy
    cf = np.clip((rh - 0.8) / 0.2, 0.0, 1.0)
    cloudy = cf > 0.0
    # column liquid / ice water paths, spread over the cloudy layers in proportion to the cloud
    # fraction times the liquid (ice) share; the layer value is the in-cloud path (g/m2)
    lwp_col = np.exp(np.log(50.0) + rng.normal(0.0, 1.0, ncol))
    iwp_col = np.exp(np.log(20.0) + rng.normal(0.0, 1.0, ncol))
    fliq = np.clip((t - 253.0) / 20.0, 0.0, 1.0)
    wl = cf * fliq
    wi = cf * (1.0 - fliq)
    sl = wl.sum(axis=0)
    si = wi.sum(axis=0)
    lwp = np.where(sl > 0, lwp_col / np.where(sl > 0, sl, 1.0), 0.0)[None, :] * np.where(wl > 0, fliq, 0.0)
    iwp = np.where(si > 0, iwp_col / np.where(si > 0, si, 1.0), 0.0)[None, :] * np.where(wi > 0, 1.0 - fliq, 0.0)

    nlay = NLEV_MODEL + 1
    plvl = np.empty((nlay + 1, ncol))
    plvl[0] = PRSMIN
    plvl[1:] = pi
    plyr = np.empty((nlay, ncol))
    plyr[0] = 0.5 * plvl[1]
    plyr[1:] = pl
    tlyr = np.empty((nlay, ncol))
    tlyr[0] = t[0]
    tlyr[1:] = t
    qlyr = np.empty((nlay, ncol))
    qlyr[0] = q[0]
    qlyr[1:] = q
    olyr = np.empty((nlay, ncol))
    o3top = 8.0e-6 * np.exp(-np.log(plyr[0] / 10.0) ** 2 / (2.0 * 1.2 ** 2)) * AMO3 / AMD
    olyr[0] = np.maximum(o3top, 0.03e-6 * AMO3 / AMD)
    olyr[1:] = o3
    tskin = tlyr[-1] + rng.normal(0.0, 3.0, ncol)
    # level temperatures: log-pressure interpolation between layer means, top = top layer, bottom = skin
    tlvl = np.empty((nlay + 1, ncol))
    tlvl[0] = tlyr[0]
    tlvl[-1] = tskin
    lpl = np.log(plvl[1:-1])
    lly = np.log(plyr)
    tlvl[1:-1] = tlyr[1:] + (tlyr[:-1] - tlyr[1:]) * (lpl - lly[1:]) / (lly[:-1] - lly[1:])

    gas = np.empty((NF_VGAS, nlay, ncol))
    for n, v in enumerate(GAS_DEFAULTS):
        gas[n] = v

    clouds = np.zeros((NF_CLDS, nlay, ncol))
    if not stress:
        clouds[0, 1:] = cf
        clouds[1, 1:] = np.where(cloudy, lwp, 0.0)
        clouds[2, 1:] = 10.0
        clouds[3, 1:] = np.where(cloudy, iwp, 0.0)
        clouds[4, 1:] = 50.0
    else:
        # diagnostic optics: tau up to 500 (log-uniform 0.1..500), ssa in [1-1e-7, 1], asymmetry 0.85
        tau = np.exp(rng.uniform(np.log(0.1), np.log(500.0), (NLEV_MODEL, ncol)))
        ssa = rng.uniform(1.0 - 1.0e-7, 1.0, (NLEV_MODEL, ncol))
        clouds[0, 1:] = cf
        clouds[1, 1:] = np.where(cloudy, tau, 0.0)
        clouds[2, 1:] = np.where(cloudy, ssa, 0.0)
        clouds[3, 1:] = np.where(cloudy, 0.85, 0.0)

    alb = rng.uniform(0.06, 0.8, ncol)
    sfcalb = np.repeat(alb[None, :], 4, axis=0)
    emis = rng.uniform(0.95, 1.0, ncol)
    if stress:
        cosz = rng.uniform(0.01, 0.05, ncol)
    else:
        cosz = rng.uniform(-1.0, 1.0, ncol)

    f = np.float32
    return Columns(plyr=plyr.astype(f), plvl=plvl.astype(f), tlyr=tlyr.astype(f), tlvl=tlvl.astype(f),
                   qlyr=qlyr.astype(f), olyr=olyr.astype(f), gasvmr=gas.astype(f),
                   clouds=clouds.astype(f), sfcemis=emis.astype(f), tsfg=tskin.astype(f),
                   sfcalb=sfcalb.astype(f), coszen=cosz.astype(f), solcon=SOLCON,
                   diagnostic_clouds=stress)


# Named workloads: (column count, seed, stress flag).
WORKLOADS = {
    "c1_plain_1024": (1024, 1001, False),
    "c2_parent_954x835": (PARENT[0] * PARENT[1], 2002, False),
    "c5_stress_200k": (200_000, 5005, True),
}


def workload(name: str, ncol: int | None = None) -> Columns:
    n, seed, stress = WORKLOADS[name]
    return make_columns(n if ncol is None else ncol, seed, stress)


def model_state(cols: "Columns") -> dict:
    """The model state a request's radiation layers come from (grrad's inputs): the lm = nlay - 1 model
    layers of the columns without the extra top layer -- interface and layer pressure in Pa, the Exner
    function (p / 1e5)^(Rd / cp), temperature, specific humidity -- and the skin temperature."""
    pmid = (cols.plyr[1:].astype(np.float64) * 100.0)
    return {"pint": (cols.plvl[1:].astype(np.float64) * 100.0).astype(np.float32),
            "pmid": pmid.astype(np.float32),
            "prslk": ((pmid / 1.0e5) ** (2.8705e2 / 1.0046e3)).astype(np.float32),
            "t": np.ascontiguousarray(cols.tlyr[1:], dtype=np.float32),
            "q": np.ascontiguousarray(cols.qlyr[1:], dtype=np.float32),
            "tsfc": np.ascontiguousarray(cols.tsfg, dtype=np.float32)}



# ---- synthetic inputs of grrad's front end (the reference's climatology files are not part of its tree) ----

OZONE_PSTR = (1.0, 2.0, 3.0, 5.0, 7.0, 10.0, 20.0, 30.0, 50.0, 70.0, 100.0, 150.0, 200.0, 300.0, 500.0, 700.0,
              1000.0)   # 17 climatology levels, hPa, top first (loz 17, as the NAM climatology)


def front_tables(seed: int = 77) -> dict:
    """Seeded stand-ins for the climatologies the front end reads, with the reference's shapes: the monthly
    15-degree CO2 map co2vmr_sav [12][12][24] with its global mean co2_glb and seasonal cycle gco2cyc [12]
    (gas_init), the ozone climatology o3r [12][17][18] on the Exner levels pkstr [17] with blte -85,
    dlte 10 (gas_init, module_SOLVER_GRID_COMP.F90 ozone settings), and the 1-degree surface-type map idxems
    [180][360] (sfc_init; values 0..9 so that the clamps of setemis are reached)."""
    r = np.random.default_rng(seed)
    lat = -85.0 + 10.0 * np.arange(18)
    lev = np.arange(17)
    prof = 2.0e-6 + 8.0e-6 * np.exp(-((lev - 6.0) / 3.5) ** 2)          # stratospheric peak
    o3r = np.empty((12, 17, 18), np.float32)
    for m in range(12):
        season = 1.0 + 0.25 * np.cos(2.0 * np.pi * (m / 12.0) + np.deg2rad(lat) * 2.0)
        o3r[m] = (prof[:, None] * season[None, :] * (1.0 + 0.05 * r.standard_normal((17, 18)))).astype(np.float32)
    pkstr = ((np.asarray(OZONE_PSTR) / 1000.0) ** (2.8705e2 / 1.0046e3)).astype(np.float32)
    return {"co2_glb": np.float32(3.95e-4),
            "gco2cyc": (3.0e-6 * np.sin(2.0 * np.pi * np.arange(12) / 12.0)).astype(np.float32),
            "co2vmr_sav": (3.95e-4 + 4.0e-6 * r.standard_normal((12, 12, 24))).astype(np.float32),
            "o3r": o3r, "pkstr": pkstr, "jmr": 18, "loz": 17, "blte": -85.0, "dlte": 10.0,
            "idxems": r.integers(0, 10, size=(180, 360)).astype(np.int32)}


def surface_state(n: int, seed: int) -> dict:
    """The surface fields setalb and setemis read, for n columns: sea / land / sea-ice masks, snow (mm, many
    columns without), roughness, orography spread, skin and ice temperatures through the freezing range, the
    four background albedos and their strong / weak zenith fractions, and the grid position."""
    r = np.random.default_rng(seed)
    f = lambda lo, hi: r.uniform(lo, hi, n).astype(np.float32)           # noqa: E731
    slmsk = r.choice(np.array([0.0, 1.0, 2.0], np.float32), n, p=[0.45, 0.45, 0.10])
    snow = np.where(r.random(n) < 0.6, 0.0, r.exponential(20.0, n)).astype(np.float32)
    cz = f(-0.3, 1.0)
    cz[r.random(n) < 0.05] = 0.0
    ts = f(235.0, 310.0)
    ts = np.where(r.random(n) < 0.2, f(270.9, 273.3), ts).astype(np.float32)
    sice = np.where(r.random(n) < 0.15, f(0.3, 1.0), 0.0).astype(np.float32)
    return {"slmsk": slmsk, "snowf": snow, "sncovr": f(0.0, 1.0), "snoalb": f(0.5, 0.85),
            "zorlf": np.exp(f(np.log(0.01), np.log(300.0))).astype(np.float32), "coszf": cz, "tsknf": ts,
            "hprif": f(0.0, 900.0), "alvsf": f(0.04, 0.35), "alnsf": f(0.05, 0.45), "alvwf": f(0.04, 0.35),
            "alnwf": f(0.05, 0.45), "facsf": f(0.0, 0.8), "facwf": f(0.0, 0.6), "fice": f(0.0, 1.0),
            "tisfc": f(245.0, 275.0),
            # setemis's names for the same kind of fields (SM: 1 sea, 0 land; Z0 in m)
            "glon": f(-np.pi, np.pi), "glat": f(-np.pi / 2, np.pi / 2),
            "sm": np.where(slmsk == 0.0, 1.0, 0.0).astype(np.float32), "sice": sice, "si": snow,
            "z0": np.exp(f(np.log(1e-4), np.log(3.0))).astype(np.float32), "stdh": f(0.0, 900.0), "tskin": ts}


def cloud_state(layers: dict, seed: int) -> dict:
    """progcld2's inputs beside the radiation layers of grrad's set-up (plyr, plvl, tlyr, tvly, qlyr, qstl, rhly
    [lmk (+1)][n], mb / K / kg/kg): total condensate clw in 0-3 decks per column (1-10 layers each, log-uniform
    1e-8..3e-4 kg/kg, so that thin, broken and overcast layers and the high / middle / low split all occur),
    the ice and rain fractions (slightly outside [0, 1] so that the clips act), the rime factor, the Thompson
    cloud fraction cldfk1 and the latitude."""
    tl = np.asarray(layers["tlyr"])
    lmk, n = tl.shape
    r = np.random.default_rng(seed)
    clw = np.zeros((lmk, n))
    ndeck = r.integers(0, 4, n)
    for d in range(3):
        has = ndeck > d
        top = r.integers(1, lmk - 1, n)
        thick = r.integers(1, 11, n)
        amt = np.exp(r.uniform(np.log(1e-8), np.log(3e-4), n))
        k = np.arange(lmk)[:, None]
        inside = has[None, :] & (k >= top[None, :]) & (k < np.minimum(top + thick, lmk)[None, :])
        clw = np.where(inside, clw + amt[None, :] * r.uniform(0.3, 1.0, (lmk, n)), clw)
    out = {k: np.ascontiguousarray(layers[k], dtype=np.float32)
           for k in ("plyr", "plvl", "tlyr", "tvly", "qlyr", "qstl", "rhly")}
    out.update({"clw": clw.astype(np.float32),
                "f_ice": r.uniform(-0.1, 1.1, (lmk, n)).astype(np.float32),
                "f_rain": r.uniform(-0.1, 1.1, (lmk, n)).astype(np.float32),
                "r_rime": r.uniform(1.0, 5.0, (lmk, n)).astype(np.float32),
                "cldfk1": np.where(clw > 0, np.clip(r.uniform(-0.2, 1.2, (lmk, n)), 0.0, 1.0), 0.0).astype(np.float32),
                "xlat": r.uniform(-np.pi / 2, np.pi / 2, n).astype(np.float32)})
    return out
