"""ctypes front end of the CPU oracle (test infrastructure only).

``liborc.so`` is the C++ restatement of the reference's RRTM LW/SW column radiation in this directory
(``rrtm_lw.hpp``, ``rrtm_sw.hpp``, ``rrtm_mcica.hpp``).  ``solve(cols, precision="double")`` returns the
same outputs as the product's C-ABI (in float64).  ``reference_solve`` runs the reference's own kernels
compiled for the host (``_ref/libref_rrtm.so``, built by ``build_ref.sh`` where the reference tree is
available) through the same interface.

Only the tests, the smoke check and the benchmark's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liborc.so"
OPCOUNT_LIB = HERE / "libopcount.so"
REF_LIB = HERE / "_ref" / "libref_rrtm.so"
TABLES = HERE.parent / "woof_nam_b200" / "data" / "rrtm_tables.npz"

_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_U = ctypes.POINTER(ctypes.c_uint)


def build(force: bool = False) -> Path:
    """Compile liborc.so and libopcount.so with the Makefile beside this file (no GPU needed)."""
    srcs = list(HERE.glob("rrtm_*.?pp")) + list(HERE.glob("opcount.hpp"))
    if force or not all(p.exists() for p in (LIB, OPCOUNT_LIB)) or any(
            p.stat().st_mtime > min(LIB.stat().st_mtime, OPCOUNT_LIB.stat().st_mtime) for p in srcs):
        subprocess.run(["make", "-C", str(HERE), *(["-B"] if force else []), "all"], check=True)
    return LIB


def _load(path: Path):
    lib = ctypes.CDLL(str(path))
    lib.orc_add_table.argtypes = [ctypes.c_char_p, _D, ctypes.c_long]
    lib.orc_add_itable.argtypes = [ctypes.c_char_p, _I, ctypes.c_long]
    if hasattr(lib, "orc_solve"):
        lib.orc_solve.restype = ctypes.c_int
    tabs = np.load(TABLES)
    lib.orc_clear_tables()
    for name in tabs.files:
        a = tabs[name]
        if a.dtype.kind == "i":
            b = np.ascontiguousarray(a, dtype=np.int32).ravel()
            lib.orc_add_itable(name.encode(), b.ctypes.data_as(_I), b.size)
        else:
            b = np.ascontiguousarray(a, dtype=np.float64).ravel()
            lib.orc_add_table(name.encode(), b.ctypes.data_as(_D), b.size)
    return lib


_LIBS: dict = {}


def lib(which: str = "port"):
    if which not in _LIBS:
        if which == "port":
            _LIBS[which] = _load(build())
        elif which == "opcount":
            build()
            _LIBS[which] = _load(OPCOUNT_LIB)
        else:
            if not REF_LIB.exists():
                raise FileNotFoundError(f"{REF_LIB} is not built (oracle/build_ref.sh needs the reference tree)")
            _LIBS[which] = _load(REF_LIB)
    return _LIBS[which]


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def solve(cols, precision: str = "double", iswmode: int = 2, window_cols: int = 0, sw_chunk: int = 32768,
          route: int = 0, iovrlw: int = 1, iovrsw: int = 1, lw_seed0: int = 140, sw_seed0: int = 1,
          cpathfac: float = 1.5, nthreads: int = 0, which: str = "port", want_profiles: bool = False,
          icseed=None, faerlw=None, faersw=None, diag: bool = False) -> dict:
    """Run the oracle on a ``woof_nam_b200.columns.Columns`` request; returns float64 outputs.  diag (the
    restatement only) adds lwrad's / swrad's optional outputs: hlw0, hlwb [16], hsw0, htswb [14] (K/s, top
    first) and the level-flux profiles lwflxprf / swflxprf [4][nlay+1] (up total, down total, up clear, down
    clear, top first)."""
    L = lib(which)
    nlay, ncol = cols.nlay, cols.ncol
    cfg = np.array([iswmode, int(cols.diagnostic_clouds), window_cols, sw_chunk, route, iovrlw, iovrsw,
                    lw_seed0, sw_seed0], dtype=np.int32)
    out = {
        "htlw": np.zeros((nlay, ncol)), "htsw": np.zeros((nlay, ncol)),
        "topflw": np.zeros((2, ncol)), "sfcflw": np.zeros((4, ncol)),
        "topfsw": np.zeros((3, ncol)), "sfcfsw": np.zeros((4, ncol)), "fdncmp": np.zeros((6, ncol)),
    }
    if want_profiles or diag:
        out["lwflx"] = np.zeros((4, nlay + 1, ncol))
        out["swflx"] = np.zeros((4, nlay + 1, ncol))
    if diag:
        if which != "port":
            raise ValueError("diag outputs come from the restatement (which='port')")
        out["hlw0"] = np.zeros((nlay, ncol))
        out["hlwb"] = np.zeros((16, nlay, ncol))
        out["hsw0"] = np.zeros((nlay, ncol))
        out["htswb"] = np.zeros((14, nlay, ncol))
    if route == 1:
        out["lw_mask"] = np.zeros((5, nlay, ncol), dtype=np.uint32)
        out["sw_mask"] = np.zeros((4, nlay, ncol), dtype=np.uint32)
    keep = [_f(getattr(cols, f)) for f in cols.FIELDS]
    fa = _f(faerlw) if faerlw is not None else None
    fs = _f(faersw) if faersw is not None else None
    seeds = np.ascontiguousarray(icseed, dtype=np.int32) if icseed is not None else None

    def p(a, t):
        return a.ctypes.data_as(t) if a is not None else None

    args = [ctypes.c_int(0 if precision == "float" else 1), p(cfg, _I), ctypes.c_double(cpathfac),
            ctypes.c_int(nlay), ctypes.c_int(ncol),
            *[p(a, _F) for a in keep[:8]], p(fa, _F), p(fs, _F), *[p(a, _F) for a in keep[8:]],
            p(seeds, _I), ctypes.c_double(cols.solcon),
            p(out["htlw"], _D), p(out["htsw"], _D), p(out["topflw"], _D), p(out["sfcflw"], _D),
            p(out["topfsw"], _D), p(out["sfcfsw"], _D), p(out["fdncmp"], _D),
            p(out.get("lwflx"), _D), p(out.get("swflx"), _D), p(out.get("lw_mask"), _U), p(out.get("sw_mask"), _U)]
    if diag:
        rc = L.orc_solve_diag(*args, p(out["hlw0"], _D), p(out["hlwb"], _D), p(out["hsw0"], _D),
                              p(out["htswb"], _D), ctypes.c_int(nthreads))
        out["lwflxprf"], out["swflxprf"] = out["lwflx"], out["swflx"]
    else:
        rc = L.orc_solve(*args, ctypes.c_int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle solve failed ({rc})")
    return out


def reference_solve(cols, **kw) -> dict:
    """The reference's own kernels compiled for the host, driven in the reference's call order (float32)."""
    kw = dict(kw)
    kw.pop("precision", None)
    return solve(cols, precision="float", which="ref", **kw)


def host_threads() -> int:
    return len(os.sched_getaffinity(0))


def set_debug(sw_tau_scale: float = 1.0, which: str = "port") -> None:
    """Test hook: scale the SW gas optical depths before the two-stream solver (1.0 = off)."""
    lib(which).orc_set_debug(ctypes.c_double(sw_tau_scale))


def sw_stages(cols, which: str = "port", iswmode: int = 2, iovrsw: int = 1) -> dict:
    """SW stage outputs (float statements) of the request's day columns, layers surface first; iovrsw is the
    overlap of the clear-sky view fraction zcf (0 random, 1 maximum-random, 2 maximum)."""
    L = lib(which)
    nlay, ncol = cols.nlay, cols.ncol
    nday = int((cols.coszen >= np.float32(1e-4)).sum())
    out = {"taug": np.zeros((nday, nlay, 112), np.float32), "taur": np.zeros((nday, nlay, 112), np.float32),
           "sfluxzen": np.zeros((nday, 112), np.float32), "taucw": np.zeros((nday, 14, nlay), np.float32),
           "ssacw": np.zeros((nday, 14, nlay), np.float32), "asycw": np.zeros((nday, 14, nlay), np.float32),
           "cldfrc": np.zeros((nday, nlay), np.float32), "zcf": np.zeros((nday, 2), np.float32),
           "laytrop": np.zeros(nday, np.int32)}
    cfg = np.array([iswmode, int(cols.diagnostic_clouds), iovrsw], dtype=np.int32)
    keep = {f: _f(getattr(cols, f)) for f in cols.FIELDS}
    rc = L.orc_sw_stages(cfg.ctypes.data_as(_I), ctypes.c_int(nlay), ctypes.c_int(ncol),
                         *[keep[f].ctypes.data_as(_F) for f in ("plyr", "plvl", "tlyr", "tlvl", "qlyr", "olyr",
                                                              "gasvmr", "clouds", "sfcalb", "coszen")],
                         ctypes.c_double(cols.solcon),
                         *[out[k].ctypes.data_as(_F) for k in ("taug", "taur", "sfluxzen", "taucw", "ssacw",
                                                              "asycw", "cldfrc", "zcf")],
                         out["laytrop"].ctypes.data_as(_I))
    if rc != 0:
        raise RuntimeError("sw_stages failed")
    return out


OPCOUNT_STAGES = ("lw_prep", "lw_cldprop", "lw_setcoef", "lw_taumol", "lw_rtrnmr",
                  "sw_prep", "sw_cldprop", "sw_setcoef", "sw_taumol", "sw_spcvrtc", "swrad_post")


def opcount(cols, iswmode: int = 2, cpathfac: float = 1.5) -> dict:
    """Operation-count table of the reference statements over the request (see opcount.hpp for the rule).

    Returns per-stage sums of (add, mul, div, func, other) and, per column, the LW FLOPs, the SW FLOPs
    per day column and the request-average FLOPs per column (LW + SW x day fraction)."""
    L = lib("opcount")
    counts = np.zeros((11, 5))
    nday = ctypes.c_int(0)
    keep = {f: _f(getattr(cols, f)) for f in cols.FIELDS}
    rc = L.orc_opcount(ctypes.c_int(int(cols.diagnostic_clouds)), ctypes.c_int(iswmode), ctypes.c_double(cpathfac),
                       ctypes.c_int(cols.nlay), ctypes.c_int(cols.ncol),
                       *[keep[f].ctypes.data_as(_F) for f in cols.FIELDS], ctypes.c_double(cols.solcon),
                       counts.ctypes.data_as(_D), ctypes.byref(nday))
    if rc != 0:
        raise RuntimeError("opcount failed")
    n, nd = cols.ncol, nday.value
    flops = counts[:, :4].sum(axis=1)
    lw = flops[:5].sum() / n
    sw = flops[5:].sum() / max(nd, 1)
    return {"stages": {s: dict(zip(("add", "mul", "div", "func", "other"), counts[i].tolist()))
                       for i, s in enumerate(OPCOUNT_STAGES)},
            "ncol": n, "nday": nd, "lw_flops_per_col": lw, "sw_flops_per_daycol": sw,
            "flops_per_col": lw + sw * nd / n}


def mcica_masks(cols, which: str = "port", iovrlw: int = 1, iovrsw: int = 1, lw_seed0: int = 140,
                sw_seed0: int = 1, icseed=None) -> dict:
    """McICA sub-column masks of a request: lw uint32 [5][nlay][ncol], sw uint32 [4][nlay][ncol], layers
    surface first (bit g & 31 of word g >> 5).  icseed: optional int32 [2][ncol] (LW row, SW row)."""
    L = lib(which)
    nlay, ncol = cols.nlay, cols.ncol
    cfg = np.array([2, 0, 0, 32768, 1, iovrlw, iovrsw, lw_seed0, sw_seed0], dtype=np.int32)
    lw = np.zeros((5, nlay, ncol), dtype=np.uint32)
    sw = np.zeros((4, nlay, ncol), dtype=np.uint32)
    cl = _f(cols.clouds)
    seeds = np.ascontiguousarray(icseed, dtype=np.int32) if icseed is not None else None
    rc = L.orc_mcica_masks(cfg.ctypes.data_as(_I), ctypes.c_int(nlay), ctypes.c_int(ncol), cl.ctypes.data_as(_F),
                           seeds.ctypes.data_as(_I) if seeds is not None else None,
                           lw.ctypes.data_as(_U), sw.ctypes.data_as(_U))
    if rc != 0:
        raise RuntimeError("mcica_masks failed")
    return {"lw": lw, "sw": sw}


# Derived aerosol tables as orc_aerosols writes them into `tab` (name, element count), in order.
AER_TAB_FIELDS = (("sigref", 35), ("extrhi", 180), ("scarhi", 180), ("ssarhi", 180), ("asyrhi", 180),
                  ("extrhd", 960), ("scarhd", 960), ("ssarhd", 960), ("asyrhd", 960), ("extstra", 30),
                  ("solbnd", 14), ("eirbnd", 16), ("cmixg", 13320), ("denng", 5328), ("idxcg", 13320),
                  ("kprfg", 2664))


def aer_climatology(month: int, path=None) -> dict:
    """The packed climatology (woof_nam_b200/data/aer_tables.npz) with one month's records (1..12)."""
    from woof_nam_b200 import aerosols
    return aerosols.climatology(month, path)


class _Flip:
    """The layer fields of a request with the vertical order reversed (plvl, plyr, tlyr, qlyr; nlay, ncol)."""

    def __init__(self, cols, fl):
        self.nlay, self.ncol = cols.nlay, cols.ncol
        for k in ("plvl", "plyr", "tlyr", "qlyr"):
            setattr(self, k, fl(getattr(cols, k)))


def aerosols(clim: dict, cols, aer_in: dict, which: str = "port", tables: bool = False, ivflip: int = 0) -> dict:
    """Aerosol optics of a request: faersw [3][14][nlay][ncol], faerlw [3][16][nlay][ncol] (float32) from the
    restatement (which="port") or the reference's kernels (which="ref"); with tables=True also the derived
    tables (AER_TAB_FIELDS).  ivflip 1: the request's layers (and the outputs') are surface first; the reference
    runs its ivflip = 1 branches, the restatement the top-first statements on the flipped layers (the reference's
    two branches mirror each other statement for statement, pinned by tests/test_aerosols.py)."""
    if ivflip == 1 and which == "port":
        fl = lambda a: np.ascontiguousarray(np.asarray(a)[::-1])  # noqa: E731
        cf = _Flip(cols, fl)
        r = aerosols(clim, cf, dict(aer_in, rhly=fl(aer_in["rhly"])), which, tables)
        for k in ("faersw", "faerlw"):
            r[k] = np.ascontiguousarray(r[k][:, :, ::-1])
        return r
    L = lib(which)
    nlay, ncol = cols.nlay, cols.ncol
    c = {k: np.ascontiguousarray(v) for k, v in clim.items()}
    ints = {k: np.ascontiguousarray(c[k], dtype=np.int32) for k in ("iendwv", "nwvns0", "month_idx", "month_kprf")}
    rhid = np.ascontiguousarray(np.stack([c["rhidext0"], c["rhidsca0"], c["rhidssa0"], c["rhidasy0"]]), np.float32)
    rhdp = np.ascontiguousarray(np.stack([c["rhdpext0"], c["rhdpsca0"], c["rhdpssa0"], c["rhdpasy0"]]), np.float32)
    f = {k: _f(c[k]) for k in ("haer", "prsref", "straext0", "s0intv")}
    d = {k: np.ascontiguousarray(c[k], dtype=np.float64) for k in ("month_cmix", "month_denn")}
    keep = [_f(getattr(cols, k)) for k in ("plvl", "plyr", "tlyr", "qlyr")] + \
           [_f(aer_in[k]) for k in ("rhly", "xlon", "xlat", "slmsk")]
    sw = np.zeros((3, 14, nlay, ncol), np.float32)
    lw = np.zeros((3, 16, nlay, ncol), np.float32)
    tab = np.zeros(sum(n for _, n in AER_TAB_FIELDS), np.float32) if tables else None
    p = lambda a, t: a.ctypes.data_as(t) if a is not None else None  # noqa: E731
    args = (p(ints["iendwv"], _I), p(f["haer"], _F), p(f["prsref"], _F), p(rhid, _F), p(rhdp, _F),
            p(f["straext0"], _F), p(ints["nwvns0"], _I), p(f["s0intv"], _F), p(ints["month_idx"], _I),
            p(d["month_cmix"], _D), p(ints["month_kprf"], _I), p(d["month_denn"], _D),
            ctypes.c_int(nlay), ctypes.c_int(ncol), *[p(a, _F) for a in keep], p(sw, _F), p(lw, _F), p(tab, _F))
    rc = L.orc_aerosols_iv(*args, ctypes.c_int(ivflip)) if ivflip else L.orc_aerosols(*args)
    if rc != 0:
        raise RuntimeError("aerosols failed")
    out = {"faersw": sw, "faerlw": lw}
    if tables:
        o = 0
        for name, n in AER_TAB_FIELDS:
            out[name] = tab[o:o + n].copy()
            o += n
    return out


def setaer_volc(plvl, xlat, ivolae, kyrsav: int, kmonsav: int, faersw, faerlw, ivflip: int = 0,
                add_sw: bool = True, add_lw: bool = True, lw1bd: bool = False, which: str = "port") -> dict:
    """setaer's volcanic stratospheric term (lavoflg) added to copies of faersw [3][14][nlay][n] and faerlw
    [3][16][nlay][n]: plvl [nlay + 1][n] mb in the order of ivflip, xlat [n] radians, ivolae int32 [10][4][12]
    (year, zone, month), kyrsav / kmonsav as the aerosol module keeps them."""
    L = lib(which)
    pl, xl = _f(plvl), _f(xlat)
    iv = np.ascontiguousarray(ivolae, dtype=np.int32)
    if iv.shape != (10, 4, 12):
        raise ValueError("ivolae must be int32 [10, 4, 12]")
    sw, lw = np.array(faersw, np.float32, copy=True, order="C"), np.array(faerlw, np.float32, copy=True, order="C")
    nlay, n = pl.shape[0] - 1, pl.shape[1]
    rc = L.orc_setaer_volc(ctypes.c_int(nlay), ctypes.c_int(n), ctypes.c_int(ivflip), _fp(pl), _fp(xl), _ip(iv),
                           ctypes.c_int(kyrsav), ctypes.c_int(kmonsav), ctypes.c_int(int(add_sw)),
                           ctypes.c_int(int(add_lw)), ctypes.c_int(int(lw1bd)), _fp(sw), _fp(lw))
    if rc != 0:
        raise ValueError("setaer_volc: invalid arguments")
    return {"faersw": sw, "faerlw": lw}


def solar(date, deltsw: float, deltim: float, solc0: float, glon=None, glat=None, solhr: float = 0.0,
          dtswav: float = 1.0, nrads: int = 1, which: str = "port") -> dict:
    """Solar geometry: sollag, sindec, cosdec, anginc, solcon, nstp of the forecast time date = (year, month,
    day, hour, minute, second), and, for columns glon / glat (radians), coszen / coszdg."""
    L = lib(which)
    d = np.ascontiguousarray(date, dtype=np.int32)
    st = np.zeros(5, np.float32)
    nstp = np.zeros(1, np.int32)
    n = 0 if glon is None else int(np.size(glon))
    lo = _f(glon if glon is not None else np.zeros(1))
    la = _f(glat if glat is not None else np.zeros(1))
    cz = np.zeros(max(n, 1), np.float32)
    cd = np.zeros(max(n, 1), np.float32)
    rc = L.orc_solar(d.ctypes.data_as(_I), ctypes.c_float(deltsw), ctypes.c_float(deltim), ctypes.c_double(solc0),
                     st.ctypes.data_as(_F), nstp.ctypes.data_as(_I), ctypes.c_int(n), lo.ctypes.data_as(_F),
                     la.ctypes.data_as(_F), ctypes.c_float(solhr), ctypes.c_float(dtswav), ctypes.c_int(nrads),
                     cz.ctypes.data_as(_F), cd.ctypes.data_as(_F))
    if rc != 0:
        raise RuntimeError("solar failed")
    out = dict(zip(("sollag", "sindec", "cosdec", "anginc", "solcon"), st.tolist()))
    out["state"] = st
    out["nstp"] = int(nstp[0])
    if n:
        out["coszen"], out["coszdg"] = cz[:n], cd[:n]
    return out


GRRAD_FIELDS = ("plvl", "plyr", "tlyr", "tlvl", "qlyr", "rhly", "qstl", "prslk1", "tvly", "tsfg")


def grrad_setup(model: dict, which: str = "port") -> dict:
    """grrad's radiation layers of a model state (pint [lm + 1][n], pmid, prslk, t, q [lm][n] in Pa / K,
    tsfc [n]): plvl, tlvl [lm + 2][n], plyr, tlyr, qlyr, rhly, qstl, prslk1, tvly [lm + 1][n], tsfg [n]."""
    L = lib(which)
    lm, n = model["pmid"].shape
    keep = [_f(model[k]) for k in ("pint", "pmid", "prslk", "t", "q", "tsfc")]
    lmk, lmp = lm + 1, lm + 2
    sizes = {"plvl": lmp, "plyr": lmk, "tlyr": lmk, "tlvl": lmp, "qlyr": lmk, "rhly": lmk, "qstl": lmk,
             "prslk1": lmk, "tvly": lmk, "tsfg": 1}
    out = np.zeros(sum(sizes.values()) * n, np.float32)
    rc = L.orc_grrad_setup(ctypes.c_int(lm), ctypes.c_int(n), *[a.ctypes.data_as(_F) for a in keep], out.ctypes.data_as(_F))
    if rc != 0:
        raise RuntimeError("grrad_setup failed")
    res, o = {}, 0
    for k in GRRAD_FIELDS:
        res[k] = out[o:o + sizes[k] * n].reshape(sizes[k], n) if k != "tsfg" else out[o:o + n]
        o += sizes[k] * n
    return res


# ---- grrad's front end (rrtm_front.hpp; which="ref": the reference's own kernels) ----

def _ip(a):
    return a.ctypes.data_as(_I)


def _fp(a):
    return a.ctypes.data_as(_F)


def _ptrs(arrs):
    """A C array of float pointers to the (kept alive) float32 copies of arrs."""
    keep = [_f(a) for a in arrs]
    return keep, (_F * len(keep))(*[_fp(a) for a in keep])


def dayparts(xlon, sinlat, coslat, im: int, solhr: float, dtswav: float, nrads: int, sol, which: str = "port") -> dict:
    """DAYPARTS of n = jm * im points (row-major): coszen, coszdg [n], the run table dp_start, dp_len, dp_day [n]
    (slot row * im + k, valid for k < ndayparts[row], others -1) and ndayparts [jm].  sol = sollag, sindec, cosdec."""
    L = lib(which)
    lo, sl, cl = _f(xlon), _f(sinlat), _f(coslat)
    n = lo.size
    jm = n // im
    s = _f(np.asarray(sol, np.float32)[:3])
    out = {"coszen": np.zeros(n, np.float32), "coszdg": np.zeros(n, np.float32)}
    for k in ("dp_start", "dp_len", "dp_day"):
        out[k] = np.full(n, -1, np.int32)
    out["ndayparts"] = np.zeros(jm, np.int32)
    L.orc_dayparts(ctypes.c_int(im), ctypes.c_int(jm), _fp(lo), _fp(sl), _fp(cl), ctypes.c_float(solhr),
                   ctypes.c_float(dtswav), ctypes.c_int(nrads), _fp(s), _fp(out["coszen"]), _fp(out["coszdg"]),
                   _ip(out["dp_start"]), _ip(out["dp_len"]), _ip(out["dp_day"]), _ip(out["ndayparts"]))
    return out


def getgases(plvl, xlon, xlat, co2_glb: float, gco2cyc, co2vmr_sav, ico2flg: int, kmonsav: int, ivflip: int,
             which: str = "port") -> np.ndarray:
    """Gas volume mixing ratios [10][lmax][n] from plvl [lmax + 1][n] (mb) and xlon / xlat [n] (radians)."""
    L = lib(which)
    pl, lo, la, cy, cs = _f(plvl), _f(xlon), _f(xlat), _f(gco2cyc), _f(co2vmr_sav)
    lmax, n = pl.shape[0] - 1, pl.shape[1]
    out = np.zeros((10, lmax, n), np.float32)
    L.orc_getgases(ctypes.c_int(n), ctypes.c_int(lmax), _fp(pl), _fp(lo), _fp(la), ctypes.c_float(co2_glb), _fp(cy),
                   _fp(cs), ctypes.c_int(ico2flg), ctypes.c_int(kmonsav), ctypes.c_int(ivflip), _fp(out))
    return out


def getozn(prslk, xlat, o3r, pkstr, k1oz: int, k2oz: int, facoz: float, blte: float, dlte: float, ivflip: int,
           init=None, which: str = "port") -> np.ndarray:
    """Ozone mass mixing ratio [nlev][n] from the Exner function prslk [nlev][n] and the climatology o3r
    [12][loz][jmr] on pkstr [loz]; levels the routine leaves alone keep init (default NaN)."""
    L = lib(which)
    pk, la, o3, ps = _f(prslk), _f(xlat), _f(o3r), _f(pkstr)
    nlev, n = pk.shape
    out = np.full((nlev, n), np.nan, np.float32) if init is None else _f(init).copy()
    L.orc_getozn(ctypes.c_int(n), ctypes.c_int(nlev), _fp(pk), _fp(la), _fp(o3), _fp(ps), ctypes.c_int(o3.shape[2]),
                 ctypes.c_int(o3.shape[1]), ctypes.c_int(k1oz), ctypes.c_int(k2oz), ctypes.c_float(facoz),
                 ctypes.c_float(blte), ctypes.c_float(dlte), ctypes.c_int(ivflip), _fp(out))
    return out


ALB_FIELDS = ("slmsk", "snowf", "sncovr", "snoalb", "zorlf", "coszf", "tsknf", "hprif", "alvsf", "alnsf", "alvwf",
              "alnwf", "facsf", "facwf", "fice", "tisfc")
EMIS_FIELDS = ("glon", "glat", "sm", "sice", "si", "sncovr", "z0", "stdh", "tskin")
CLD_FIELDS = ("plyr", "plvl", "tlyr", "tvly", "qlyr", "qstl", "rhly", "clw", "f_ice", "f_rain", "r_rime", "cldfk1",
              "xlat")
CLD_CFG = ("ivflip", "llyr", "iovr", "lcrick", "lcnorm", "lnoprec", "lsashal", "cld_fraction")


def setalb(sfc: dict, ialbflg: int, which: str = "port") -> np.ndarray:
    """Surface albedo [4][n] of the SW call from the ALB_FIELDS of sfc ([n] each)."""
    L = lib(which)
    keep, pp = _ptrs([sfc[k] for k in ALB_FIELDS])
    n = keep[0].size
    out = np.zeros((4, n), np.float32)
    L.orc_setalb(ctypes.c_int(n), pp, ctypes.c_int(ialbflg), _fp(out))
    return out


def setemis(sfc: dict, idxems, ialbflg: int, iemslw: int, which: str = "port") -> np.ndarray:
    """Surface emissivity [n] of the LW call from the EMIS_FIELDS of sfc and the type map idxems [180][360]."""
    L = lib(which)
    keep, pp = _ptrs([sfc[k] for k in EMIS_FIELDS])
    ix = np.ascontiguousarray(idxems, dtype=np.int32)
    n = keep[0].size
    out = np.zeros(n, np.float32)
    L.orc_setemis(ctypes.c_int(n), pp, _ip(ix), ctypes.c_int(ialbflg), ctypes.c_int(iemslw), _fp(out))
    return out


def grrad_clw(tracer, ntcw: int, ncld: int = 1, epsq: float = 1.0e-12, which: str = "port") -> np.ndarray:
    """grrad's condensate clw [lmk][n] from the tracers [ntrac][lmk][n]: the ncld tracers from ntcw (1-based)."""
    L = lib(which)
    tr = _f(tracer)
    ntrac, lmk, n = tr.shape
    if ntcw < 1 or ntcw - 1 + ncld > ntrac:
        raise ValueError(f"grrad_clw: tracers {ntcw}..{ntcw + ncld - 1} outside 1..{ntrac}")
    out = np.zeros((lmk, n), np.float32)
    L.orc_grrad_clw(ctypes.c_int(n), ctypes.c_int(lmk), _fp(tr), ctypes.c_int(ntcw - 1), ctypes.c_int(ncld),
                    ctypes.c_float(epsq), _fp(out))
    return out


PAYNE_OUT = ("sfcalbedo", "smx", "czmean", "alvsf", "alnsf", "alvwf", "alnwf", "facsf", "facwf")


def payne_albedo(salbedo, sm, coszen, tables: dict, which: str = "port") -> dict:
    """grrad's IALB = 2 surface albedo [n] and the fields it hands setalb (PAYNE_OUT) from salbedo, sm, coszen
    [n] and the packed tables (woof_nam_b200/data/payne_albedo.npz: trn, za, dza, albd)."""
    L = lib(which)
    a, m, c = _f(salbedo), _f(sm), _f(coszen)
    t = {k: _f(tables[k]) for k in ("trn", "za", "dza", "albd")}
    n = a.size
    out = np.zeros((9, n), np.float32)
    L.orc_payne_albedo(ctypes.c_int(n), _fp(a), _fp(m), _fp(c), _fp(t["trn"]), _fp(t["za"]), _fp(t["dza"]),
                       _fp(t["albd"]), _fp(out))
    return {k: out[i] for i, k in enumerate(PAYNE_OUT)}


def progcld2(cld: dict, cfg: dict, which: str = "port") -> dict:
    """Ferrier cloud properties of the CLD_FIELDS of cld ([nlay][n], plvl [nlay + 1][n], xlat [n]) under the
    CLD_CFG switches: clouds [9][nlay][n], clds [5][n], mtop, mbot [3][n]."""
    L = lib(which)
    keep, pp = _ptrs([cld[k] for k in CLD_FIELDS])
    nlay, n = keep[0].shape
    c = np.array([int(cfg[k]) for k in CLD_CFG], np.int32)
    out = {"clouds": np.zeros((9, nlay, n), np.float32), "clds": np.zeros((5, n), np.float32),
           "mtop": np.zeros((3, n), np.int32), "mbot": np.zeros((3, n), np.int32)}
    L.orc_progcld2(ctypes.c_int(n), ctypes.c_int(nlay), pp, _ip(c), _fp(out["clouds"]), _fp(out["clds"]),
                   _ip(out["mtop"]), _ip(out["mbot"]))
    return out
