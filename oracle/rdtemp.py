"""CPU restatement of RDTEMP, the radiative temperature change of every model step (test infrastructure
only).

Restates rdtemp_apply, namgpu/kernels/drv_rdtemp.cu:140-198 (module_RA_GFDL.F90:116-233, with ZENITH,
:1662-1805, and CAL_MON_DAY, :7823-7856), in numpy float32: the step's solar declination and hour angle,
the zenith cosine CZEN on the tile, and T += (RSWTT x CZEN / CZMEAN + RLWTT) x DT on the interior.
``reference_rdtemp`` runs the reference kernel itself, compiled for the host into ``_ref/libref_rrtm.so``.
Transcendentals (sin, asin, acos, cos) come from numpy here and from the device / host libm there, so the
three agree to float rounding, not to the bit.

Only the tests and the fixture script import this module.
"""
from __future__ import annotations

import ctypes

import numpy as np

f32 = np.float32
MONTH = (31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31)
# 1-based slots of the loop-limit table the reference kernel reads (nmmb_common.cuh DL_*)
DL = {"its": 4, "ite": 5, "jts": 6, "jte": 7, "its_b1": 8, "ite_b1": 9, "jts_b1": 12, "jte_b1": 13}


def _mdays(year: int, leap_seen: int) -> list:
    m = list(MONTH)
    if year % 4 == 0 or leap_seen:
        m[1] = 29
    return m


def sun(ntsd: int, dt: float, julday: int, julyr: int, ihrst: int, leap_seen: int) -> tuple:
    """(dec, hrang) of the step, float32 (ZENITH's scalar part after CAL_MON_DAY)."""
    pi = f32(3.1415926)
    twopi = f32(2.0) * pi
    d2r = f32(3.1415926) / f32(180.0)
    month = _mdays(julyr, leap_seen)
    left, mon, mday = julday, 12, julday
    for m in range(12):
        if left > month[m]:
            left -= month[m]
        else:
            mday, mon = left, m + 1
            break
    times = f32(ntsd) * f32(dt)
    day = f32(0.0)
    for m in range(mon - 1):
        day = f32(day + f32(month[m]))
    day = f32(day + f32(mday - 1) + (f32(ihrst) + times / f32(3600.0)) / f32(24.0))
    dayi = f32(int(day) + 1)
    hour = f32((day - dayi + f32(1.0)) * f32(24.0))
    yfctr = f32(2000.0) - f32(julyr)
    dy = julyr - 2000
    addday = f32(int(dy / 4)) if dy < 0 else f32((dy + 3) // 4)
    startyr = f32(f32(2451545.0) + f32(dy) * f32(365.0) + addday - f32(0.5))
    difjd = f32(startyr + day - f32(2451545.0))
    slonm = f32((f32(280.460) + f32(0.9856474) * difjd) * d2r + yfctr * twopi)
    anom = f32((f32(357.528) + f32(0.9856003) * difjd) * d2r)
    slon = f32(slonm + (f32(1.915) * np.sin(anom) + f32(0.020) * np.sin(f32(2.0) * anom)) * d2r)
    if slon > twopi:
        slon = f32(slon - twopi)
    dec = f32(np.arcsin(f32(np.sin(slon) * np.sin(f32(23.440) * d2r))))
    ra = f32(np.arccos(f32(np.cos(slon) / np.cos(dec))))
    if slon > pi:
        ra = f32(twopi - ra)
    tu = f32((startyr + dayi - f32(1.0) - f32(2451545.0)) / f32(36525.0))
    stim0 = f32(f32(24110.54841) + tu * (f32(8640184.812866) + f32(9.3104e-2) * tu + f32(-6.2e-6) * tu * tu))
    sidtim = f32((stim0 / f32(3600.0) + yfctr * f32(24.0) + f32(1.00273791) * hour) * f32(15.0) * d2r)
    if sidtim < 0:
        sidtim = f32(sidtim + twopi)
    if sidtim > twopi:
        sidtim = f32(sidtim - twopi)
    return dec, f32(sidtim - ra)


def rdtemp(p: dict) -> dict:
    """p: ntsd, dt, julday, julyr, ihrst, leap_seen, glat, glon, czmean [jm, im], rswtt, rlwtt, t
    [lm, jm, im], czen (values kept outside the tile), limits its..jte_b1 (1-based).  Returns czen, t."""
    dec, hrang = sun(p["ntsd"], p["dt"], p["julday"], p["julyr"], p["ihrst"], p["leap_seen"])
    jm, im = p["glat"].shape
    czen = p["czen"].astype(f32, copy=True)
    t = p["t"].astype(f32, copy=True)
    jj, ii = np.meshgrid(np.arange(jm), np.arange(im), indexing="ij")
    tile = (ii >= p["its"] - 1) & (ii <= p["ite"] - 1) & (jj >= p["jts"] - 1) & (jj <= p["jte"] - 1)
    inner = tile & (ii >= p["its_b1"] - 1) & (ii <= p["ite_b1"] - 1) & (jj >= p["jts_b1"] - 1) & (jj <= p["jte_b1"] - 1)
    lat, lon = p["glat"].astype(f32), p["glon"].astype(f32)
    hrlcl = (hrang + lon + f32(2.0) * f32(3.1415926)).astype(f32)
    sinalt = (np.sin(dec) * np.sin(lat) + np.cos(dec) * np.cos(hrlcl) * np.cos(lat)).astype(f32)
    sinalt = np.maximum(sinalt, f32(0.0))
    czen[tile] = sinalt[tile]
    cm = p["czmean"].astype(f32)
    factr = np.where(cm > 0, sinalt / np.where(cm > 0, cm, f32(1.0)), f32(0.0)).astype(f32)
    tend = (p["rswtt"].astype(f32) * factr + p["rlwtt"].astype(f32)).astype(f32)
    t = np.where(inner[None], (t + tend * f32(p["dt"])).astype(f32), t)
    return {"czen": czen, "t": t}


def reference_rdtemp(p: dict) -> dict:
    """The reference kernel rdtemp_apply on the host (oracle/_ref)."""
    from . import oracle
    lib = ctypes.CDLL(str(oracle.REF_LIB))
    jm, im = p["glat"].shape
    lm = p["t"].shape[0]
    c = lambda a: np.ascontiguousarray(a, dtype=f32)  # noqa: E731
    glat, glon, czm, rsw, rlw = c(p["glat"]), c(p["glon"]), c(p["czmean"]), c(p["rswtt"]), c(p["rlwtt"])
    czen, t = c(p["czen"]).copy(), c(p["t"]).copy()
    lim = np.zeros(32, dtype=np.int32)
    for k, slot in DL.items():
        lim[slot] = p[k]
    fp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    lib.ref_rdtemp(ctypes.c_int(p["ntsd"]), ctypes.c_float(p["dt"]), ctypes.c_int(p["julday"]), ctypes.c_int(p["julyr"]),
                   ctypes.c_int(p["ihrst"]), ctypes.c_int(p["leap_seen"]), fp(glat), fp(glon), fp(czen), fp(czm),
                   fp(t), fp(rsw), fp(rlw), ctypes.c_int(im), ctypes.c_int(jm), ctypes.c_int(lm), fp(lim))
    return {"czen": czen, "t": t}


def make_case(im: int, jm: int, lm: int, seed: int, ntsd: int = 37, julday: int = 73, julyr: int = 2025,
              ihrst: int = 12) -> dict:
    """Seeded RDTEMP inputs on an im x jm grid: latitudes / longitudes of a regional domain, mean zenith
    cosines (a quarter of them zero), heating rates, temperatures; the tile is the whole grid and the
    interior drops one row / column at each edge (ITS_B1 = 2, ITE_B1 = IM - 1)."""
    rng = np.random.default_rng(seed)
    lat = np.deg2rad(np.linspace(10, 60, jm))[:, None] + np.zeros((1, im))
    lon = np.deg2rad(np.linspace(-130, -60, im))[None, :] + np.zeros((jm, 1))
    czm = rng.uniform(0, 1, (jm, im))
    czm[rng.random((jm, im)) < 0.25] = 0.0
    return {"ntsd": ntsd, "dt": 9.0, "julday": julday, "julyr": julyr, "ihrst": ihrst, "leap_seen": int(julyr % 4 == 0),
            "glat": lat.astype(f32), "glon": lon.astype(f32), "czmean": czm.astype(f32),
            "rswtt": rng.uniform(0, 3e-4, (lm, jm, im)).astype(f32), "rlwtt": rng.uniform(-3e-4, 1e-4, (lm, jm, im)).astype(f32),
            "t": rng.uniform(190, 310, (lm, jm, im)).astype(f32), "czen": np.full((jm, im), -1.0, f32),
            "its": 1, "ite": im, "jts": 1, "jte": jm, "its_b1": 2, "ite_b1": im - 1, "jts_b1": 2, "jte_b1": jm - 1}
