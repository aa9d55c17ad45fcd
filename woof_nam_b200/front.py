"""grrad's front end on the GPU: the column solve's inputs from the model state, the surface fields and the
climatologies, one library kernel per routine (rad_dayparts, rad_getgases, rad_getozn, rad_setalb, rad_setemis,
rad_progcld2).  The functions mirror the reference's units (namgpu/physics/rrtm/phys_rrtm_dayparts.py,
phys_rrtm_getgases.py, phys_rrtm_getozn.py, phys_rrtm_setalb.py, phys_rrtm_setemis.py, phys_rrtm_progcld2.py):
the same names, argument meaning and checks, with CUDA float32 tensors in the solve's layout ([field][level]
[column], column = row * im + point) where the reference takes CuPy arrays [.., JM, IM].

    from woof_nam_b200 import front
    dp = front.dayparts(solver, glon, torch.sin(glat), torch.cos(glat), solhr, dtswav, nrads, sun, im)
    gas = front.getgases(solver, lay["plvl"], glon, glat, gasvmr, co2_glb=..., gco2cyc=..., co2vmr_sav=...,
                         ico2flg=1, kmonsav=7, ivflip=0)

Every function launches on the given stream (default: torch's current one) and returns its outputs; nothing
is read back to the host.
"""
from __future__ import annotations

import ctypes
import functools

from . import _lib

NF_VGAS = 10
NF_CLDS = 9
NF_ALBD = 4


def _torch():
    import torch
    return torch


def _dev(t, name: str, unit: str, dtype=None):
    torch = _torch()
    dtype = dtype or torch.float32
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise TypeError(f"{unit}: {name} must be a contiguous {dtype} CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


def _chk(t, name: str, unit: str, shape: tuple, dtype=None):
    """t must be a contiguous CUDA tensor of `dtype` (float32 by default) and `shape` (the kernels index by the
    sizes passed beside the pointers, so a mismatch is refused here, before any launch)."""
    _dev(t, name, unit, dtype)
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{unit}: {name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t


def _stream(stream):
    torch = _torch()
    return ctypes.c_void_p((stream if stream is not None else torch.cuda.current_stream()).cuda_stream)


def _ptr(t):
    return None if t is None else t.data_ptr()


def dayparts(solver, xlon, sinlat, coslat, solhr: float, dtswav: float, nrads: int, sun: dict, im: int,
             out: dict | None = None, stream=None) -> dict:
    """DAYPARTS of n = jm * im points (phys_rrtm_dayparts.dayparts): coszen, coszdg [n], the run table dp_start,
    dp_len, dp_day [n] (run k of row j in slot j * im + k, valid for k < ndayparts[j]) and ndayparts [jm].  sun is
    solar.sol_update's dict (sollag, sindec, cosdec)."""
    torch = _torch()
    n = xlon.numel()
    if im < 1 or n % im != 0:
        raise ValueError(f"dayparts: n={n} is not a whole number of rows of im={im}")
    jm = n // im
    if out is None:
        dev = xlon.device
        out = {"coszen": torch.empty(n, dtype=torch.float32, device=dev),
               "coszdg": torch.empty(n, dtype=torch.float32, device=dev)}
        for k in ("dp_start", "dp_len", "dp_day"):
            out[k] = torch.zeros(n, dtype=torch.int32, device=dev)
        out["ndayparts"] = torch.zeros(jm, dtype=torch.int32, device=dev)
    for k in ("xlon", "sinlat", "coslat"):
        _chk({"xlon": xlon, "sinlat": sinlat, "coslat": coslat}[k], k, "dayparts", (n,))
    for k in _lib.DAYPARTS_FIELDS:
        _chk(out[k], k, "dayparts", (jm,) if k == "ndayparts" else (n,),
             torch.float32 if k in ("coszen", "coszdg") else torch.int32)
    o = _lib.RadDayparts(*[_ptr(out[k]) for k in _lib.DAYPARTS_FIELDS])
    args = [_dev(t, k, "dayparts") for k, t in (("xlon", xlon), ("sinlat", sinlat), ("coslat", coslat))]
    rc = solver.lib.rad_dayparts(solver.handle, ctypes.byref(sun["_state"]), *args, int(im), int(jm), float(solhr),
                                 float(dtswav), int(nrads), ctypes.byref(o), _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_dayparts")
    return out


def getgases(solver, plvl, xlon, xlat, gasvmr=None, *, co2_glb, gco2cyc, co2vmr_sav, ico2flg: int, kmonsav,
             ivflip: int, stream=None):
    """Gas volume mixing ratios gasvmr [10][lmax][n] (phys_rrtm_getgases.getgases) from plvl [lmax + 1][n] (mb),
    xlon, xlat [n]; co2_glb [1], gco2cyc [12], co2vmr_sav [12][12][24] device tensors (gas_init's)."""
    torch = _torch()
    lmax, n = plvl.shape[0] - 1, plvl.shape[1]
    if gasvmr is None:
        gasvmr = torch.empty((NF_VGAS, lmax, n), dtype=torch.float32, device=plvl.device)
    if tuple(gasvmr.shape) != (NF_VGAS, lmax, n):
        raise ValueError(f"getgases: gasvmr shape {tuple(gasvmr.shape)} does not match [10, {lmax}, {n}]")
    _chk(xlon, "xlon", "getgases", (n,))
    _chk(xlat, "xlat", "getgases", (n,))
    for k, t, m in (("co2_glb", co2_glb, 1), ("gco2cyc", gco2cyc, 12), ("co2vmr_sav", co2vmr_sav, 12 * 12 * 24)):
        if t is not None:
            _chk(t.reshape(-1) if t.is_contiguous() else t, k, "getgases", (m,))
    g = _lib.RadGasSetup(_ptr(co2_glb), _ptr(gco2cyc), _ptr(co2vmr_sav), int(ico2flg),
                         int(kmonsav) if kmonsav is not None else 0, int(ivflip))
    rc = solver.lib.rad_getgases(solver.handle, _dev(plvl, "plvl", "getgases"), _dev(xlon, "xlon", "getgases"),
                                 _dev(xlat, "xlat", "getgases"), n, lmax, ctypes.byref(g),
                                 _dev(gasvmr, "gasvmr", "getgases"), _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_getgases")
    return gasvmr


def getozn(solver, prslk, xlat, o3mmr=None, *, o3r, pkstr, k1oz: int, k2oz: int, facoz: float, blte: float,
           dlte: float, ivflip: int = 0, stream=None):
    """Climatological ozone o3mmr [nlev][n] (phys_rrtm_getozn) from the Exner function prslk [nlev][n] and xlat
    [n]; o3r [12][loz][jmr], pkstr [loz] device tensors, k1oz / k2oz / facoz from gas_update."""
    torch = _torch()
    nlev, n = prslk.shape
    if o3mmr is None:
        o3mmr = torch.zeros((nlev, n), dtype=torch.float32, device=prslk.device)
    _chk(xlat, "xlat", "getozn", (n,))
    _chk(o3mmr, "o3mmr", "getozn", (nlev, n))
    if o3r.dim() != 3 or o3r.shape[0] != 12:
        raise ValueError(f"getozn: o3r must be [12, loz, jmr], got {tuple(o3r.shape)}")
    _chk(o3r, "o3r", "getozn", tuple(o3r.shape))
    _chk(pkstr, "pkstr", "getozn", (int(o3r.shape[1]),))
    c = _lib.RadOzoneClim(_ptr(o3r), _ptr(pkstr), int(o3r.shape[2]), int(o3r.shape[1]), int(k1oz), int(k2oz),
                          float(facoz), float(blte), float(dlte), int(ivflip))
    rc = solver.lib.rad_getozn(solver.handle, _dev(prslk, "prslk", "getozn"), _dev(xlat, "xlat", "getozn"), n, nlev,
                               ctypes.byref(c), _dev(o3mmr, "o3mmr", "getozn"), _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_getozn")
    return o3mmr


def setalb(solver, sfc: dict, ialbflg: int, sfcalb=None, stream=None):
    """Surface albedo sfcalb [4][n] (phys_rrtm_setalb) from the ALBEDO_FIELDS of sfc ([n] CUDA tensors; zorlf in
    cm, snowf in mm).  ialbflg 2 reads only alvsf, alnsf, alvwf, alnwf."""
    torch = _torch()
    n = sfc["alvsf"].numel()
    if sfcalb is None:
        sfcalb = torch.empty((NF_ALBD, n), dtype=torch.float32, device=sfc["alvsf"].device)
    for k in _lib.ALBEDO_FIELDS:
        if sfc.get(k) is not None:
            _chk(sfc[k], k, "setalb", (n,))
    _chk(sfcalb, "sfcalb", "setalb", (NF_ALBD, n))
    a = _lib.RadAlbedoIn(*[_ptr(sfc.get(k)) for k in _lib.ALBEDO_FIELDS])
    rc = solver.lib.rad_setalb(solver.handle, ctypes.byref(a), n, int(ialbflg), _dev(sfcalb, "sfcalb", "setalb"),
                               _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_setalb")
    return sfcalb


def setemis(solver, sfc: dict, idxems, ialbflg: int, iemslw: int, sfcemis=None, stream=None):
    """Surface emissivity sfcemis [n] (phys_rrtm_setemis) from glon, glat, sm, sice, si, sncovr, z0, stdh, tskin
    [n] of sfc and the int32 type map idxems [180][360]."""
    torch = _torch()
    n = sfc["glon"].numel()
    if sfcemis is None:
        sfcemis = torch.empty(n, dtype=torch.float32, device=sfc["glon"].device)
    if idxems is not None:
        _chk(idxems, "idxems", "setemis", (180, 360), torch.int32)
    for k in _lib.EMIS_FIELDS[:-1]:
        if sfc.get(k) is not None:
            _chk(sfc[k], k, "setemis", (n,))
    _chk(sfcemis, "sfcemis", "setemis", (n,))
    vals = [_ptr(sfc.get(k)) for k in _lib.EMIS_FIELDS[:-1]] + [_ptr(idxems)]
    e = _lib.RadEmisIn(*vals)
    rc = solver.lib.rad_setemis(solver.handle, ctypes.byref(e), n, int(ialbflg), int(iemslw),
                                _dev(sfcemis, "sfcemis", "setemis"), _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_setemis")
    return sfcemis


def progcld2(solver, inputs: dict, *, ivflip: int, llyr: int, iovr: int, lcrick: bool = False, lcnorm: bool = False,
             lnoprec: bool = False, lsashal: bool = False, cld_fraction: int = 0, out: dict | None = None,
             stream=None) -> dict:
    """Ferrier cloud properties (phys_rrtm_progcld2.run) of the CLOUD_IN_FIELDS of inputs: clouds [9][nlay][n],
    clds [5][n], mtop, mbot [3][n] (1-based layers) -- the dict keys the reference's unit returns as clouds,
    clds, mtopa, mbota."""
    torch = _torch()
    nlay, n = inputs["plyr"].shape
    if cld_fraction != 0 and inputs.get("cldfk1") is None:
        raise RuntimeError(f"progcld2: cld_fraction={cld_fraction} needs cldfk1 (Thompson)")
    if out is None:
        dev = inputs["plyr"].device
        out = {"clouds": torch.empty((NF_CLDS, nlay, n), dtype=torch.float32, device=dev),
               "clds": torch.empty((5, n), dtype=torch.float32, device=dev),
               "mtop": torch.empty((3, n), dtype=torch.int32, device=dev),
               "mbot": torch.empty((3, n), dtype=torch.int32, device=dev)}
    for k in _lib.CLOUD_IN_FIELDS:
        if inputs.get(k) is not None:
            _chk(inputs[k], k, "progcld2", (nlay + 1, n) if k == "plvl" else (n,) if k == "xlat" else (nlay, n))
    for k, shape, dt in (("clouds", (NF_CLDS, nlay, n), torch.float32), ("clds", (5, n), torch.float32),
                         ("mtop", (3, n), torch.int32), ("mbot", (3, n), torch.int32)):
        _chk(out[k], k, "progcld2", shape, dt)
    ci = _lib.RadCloudIn(*[_ptr(inputs.get(k)) for k in _lib.CLOUD_IN_FIELDS])
    cfg = _lib.RadCloudCfg(int(ivflip), int(llyr), int(iovr), int(bool(lcrick)), int(bool(lcnorm)), int(bool(lnoprec)),
                           int(bool(lsashal)), int(cld_fraction))
    co = _lib.RadCloudOut(*[_ptr(out[k]) for k in _lib.CLOUD_OUT_FIELDS])
    rc = solver.lib.rad_progcld2(solver.handle, ctypes.byref(ci), n, nlay, ctypes.byref(cfg), ctypes.byref(co),
                                 _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_progcld2")
    out["mtopa"], out["mbota"] = out["mtop"], out["mbot"]
    return out


def grrad_clw(solver, tracer, ntcw: int, ncld: int = 1, clw=None, epsq: float = 1.0e-12, stream=None):
    """grrad's condensate clw [lmk][n] (phys_rrtm_grrad_clouds: grrad_clouds_clw) from the tracers [ntrac][lmk][n]:
    the ncld tracers from ntcw (1-based; NAM ncld 1) summed, below epsq zero."""
    torch = _torch()
    if tracer.dim() != 3:
        raise ValueError(f"grrad_clw: tracer must be [ntrac, lmk, n], got {tuple(tracer.shape)}")
    ntrac, lmk, n = tracer.shape
    _chk(tracer, "tracer", "grrad_clw", (ntrac, lmk, n))
    if clw is None:
        clw = torch.empty((lmk, n), dtype=torch.float32, device=tracer.device)
    _chk(clw, "clw", "grrad_clw", (lmk, n))
    rc = solver.lib.rad_grrad_clw(solver.handle, _dev(tracer, "tracer", "grrad_clw"), int(ntrac), int(lmk), int(n),
                                  int(ntcw), int(ncld), float(epsq), _dev(clw, "clw", "grrad_clw"), _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_grrad_clw")
    return clw


PAYNE_OUT = ("sfcalbedo", "smx", "czmean", "alvsf", "alnsf", "alvwf", "alnwf", "facsf", "facwf")


@functools.lru_cache(maxsize=4)
def payne_tables(path=None) -> dict:
    """The IALB = 2 albedo tables (trn, za, dza, albd) as float32 numpy arrays (woof_nam_b200/data/payne_albedo.npz)."""
    import numpy as np
    from pathlib import Path
    p = Path(path) if path is not None else Path(__file__).resolve().parent / "data" / "payne_albedo.npz"
    with np.load(p) as z:
        return {k: np.ascontiguousarray(z[k], dtype=np.float32) for k in ("trn", "za", "dza", "albd")}


def payne_albedo(solver, salbedo, sm, coszen, tables: dict | None = None, out: dict | None = None, stream=None):
    """grrad's IALB = 2 surface albedo (phys_rrtm_grrad_clouds: grrad_clouds_albedo) of n points from salbedo, sm,
    coszen [n]: a dict of PAYNE_OUT [n] CUDA tensors, alvsf / alnsf / alvwf / alnwf / facsf / facwf being what
    setalb (ialbflg 2) reads."""
    import numpy as np
    torch = _torch()
    n = salbedo.numel()
    for k, t in (("salbedo", salbedo), ("sm", sm), ("coszen", coszen)):
        _chk(t, k, "payne_albedo", (n,))
    t = tables if tables is not None else payne_tables()
    sizes = {"trn": (21,), "za": (20,), "dza": (19,), "albd": (20, 21)}
    arr = {k: np.ascontiguousarray(t[k], dtype=np.float32) for k in sizes}
    for k, shp in sizes.items():
        if arr[k].shape != shp:
            raise ValueError(f"payne_albedo: table {k} has shape {arr[k].shape}, expected {shp}")
    if out is None:
        out = {k: torch.empty(n, dtype=torch.float32, device=salbedo.device) for k in PAYNE_OUT}
    for k in PAYNE_OUT:
        _chk(out[k], k, "payne_albedo", (n,))
    fp = ctypes.POINTER(ctypes.c_float)
    tb = _lib.RadPayneTables(*[arr[k].ctypes.data_as(fp) for k in ("trn", "za", "dza", "albd")])
    ptrs = (ctypes.c_void_p * 9)(*[out[k].data_ptr() for k in PAYNE_OUT])
    rc = solver.lib.rad_payne_albedo(solver.handle, _dev(salbedo, "salbedo", "payne_albedo"),
                                     _dev(sm, "sm", "payne_albedo"), _dev(coszen, "coszen", "payne_albedo"), int(n),
                                     ctypes.byref(tb), ptrs, _stream(stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_payne_albedo")
    return out
