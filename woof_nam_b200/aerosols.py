"""Climatological aerosol optics of the NAM radiation (setaer / aer_property, iaer = 11) on the GPU.

The monthly 5-degree OPAC climatology and its optical tables (``data/aer_tables.npz``, packed from the NAM
data file) are turned into the band tables once per month by the library (``rad_load_aerosols``: the solar
and IR spectra of set_spectrum, the band weights and averages of clim_aerinit, the month's fill of
aer_update), and every radiation step maps them onto the columns (``rad_setaer``: setaer's layer
thicknesses and heights, aer_property's profile choice, humidity interpolation and smoothing), giving the
``faersw [3][14][nlay][ncol]`` / ``faerlw [3][16][nlay][ncol]`` (optical depth, single-scattering albedo,
asymmetry per band) that rad_solve takes as RadColumns.faersw / faerlw.

    from woof_nam_b200.aerosols import Aerosols, climatology
    aer = Aerosols(solver, month=7)                    # tables of July on the solver's device
    fsw, flw = aer.optics(dev, rhly, xlon, xlat, slmsk) # device tensors for rad_solve

Inputs follow the radiation arrays (top first, levels [nlay + 1][ncol], layers [nlay][ncol]); longitude and
latitude in radians (the grid's XLON / XLAT), the sea-land mask SLMSK (0 sea, 1 land, 2 sea ice) and the
layer relative humidity (grrad's RHLY, 0..1).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

NPZ = Path(__file__).resolve().parent / "data" / "aer_tables.npz"
OPTICAL = ("iendwv", "haer", "prsref", "rhidext0", "rhidsca0", "rhidssa0", "rhidasy0", "rhdpext0", "rhdpsca0",
           "rhdpssa0", "rhdpasy0", "straext0", "nwvns0", "s0intv")
MONTHLY = ("month_idx", "month_cmix", "month_kprf", "month_denn")


def climatology(month: int, path=None) -> dict:
    """The optical tables and the records of one month (1..12) of the packed climatology."""
    if not 1 <= int(month) <= 12:
        raise ValueError(f"month {month} is not 1..12")
    z = np.load(path or NPZ)
    out = {k: z[k] for k in OPTICAL}
    for k in MONTHLY:
        out[k] = z[k][int(month) - 1]
    return out


def relative_humidity(cols) -> np.ndarray:
    """Layer relative humidity [nlay][ncol] of a column request, from specific humidity over water saturation
    (Bolton's formula), clipped to 0..1 -- a stand-in for grrad's RHLY in synthetic requests."""
    t = cols.tlyr.astype(np.float64)
    p = cols.plyr.astype(np.float64)
    es = np.minimum(6.112 * np.exp(17.67 * (t - 273.15) / (t - 29.65)), 0.5 * p)
    qs = 0.622 * es / (p - 0.378 * es)
    return np.clip(cols.qlyr / qs, 0.0, 1.0).astype(np.float32)


def make_inputs(cols, seed: int, region: str = "nam") -> dict:
    """Seeded aerosol inputs for a column request: rhly from the columns, longitude / latitude in radians over
    the NAM domain (region "nam": 10..60 N, 130..60 W) or the whole globe ("globe"), and a land mask."""
    rng = np.random.default_rng(seed)
    n = cols.ncol
    if region == "nam":
        lon = rng.uniform(-130.0, -60.0, n)
        lat = rng.uniform(10.0, 60.0, n)
    else:
        lon = rng.uniform(-180.0, 360.0, n)
        lat = rng.uniform(-90.0, 90.0, n)
    slm = rng.choice(np.array([0.0, 1.0, 2.0]), size=n, p=[0.5, 0.45, 0.05])
    return {"rhly": relative_humidity(cols), "xlon": np.deg2rad(lon).astype(np.float32),
            "xlat": np.deg2rad(lat).astype(np.float32), "slmsk": slm.astype(np.float32)}


def _clim_struct(clim: dict):
    """RadAerClim over host arrays (kept alive by the returned list)."""
    import ctypes

    from . import _lib
    keep = {
        "iendwv": np.ascontiguousarray(clim["iendwv"], np.int32),
        "haer": np.ascontiguousarray(clim["haer"], np.float32),
        "prsref": np.ascontiguousarray(clim["prsref"], np.float32),
        "rhid": np.ascontiguousarray(np.stack([clim[k] for k in ("rhidext0", "rhidsca0", "rhidssa0", "rhidasy0")]), np.float32),
        "rhdp": np.ascontiguousarray(np.stack([clim[k] for k in ("rhdpext0", "rhdpsca0", "rhdpssa0", "rhdpasy0")]), np.float32),
        "straext0": np.ascontiguousarray(clim["straext0"], np.float32),
        "nwvns0": np.ascontiguousarray(clim["nwvns0"], np.int32),
        "s0intv": np.ascontiguousarray(clim["s0intv"], np.float32),
        "month_idx": np.ascontiguousarray(clim["month_idx"], np.int32),
        "month_cmix": np.ascontiguousarray(clim["month_cmix"], np.float64),
        "month_kprf": np.ascontiguousarray(clim["month_kprf"], np.int32),
        "month_denn": np.ascontiguousarray(clim["month_denn"], np.float64),
    }
    c = _lib.RadAerClim()
    for k in _lib.AER_CLIM_FIELDS:
        setattr(c, k, keep[k].ctypes.data_as(ctypes.c_void_p))
    return c, keep


class Aerosols:
    """The aerosol optics of a solver's handle: load a month's climatology, then optics() per radiation step."""

    def __init__(self, solver, month: int, clim: dict | None = None):
        self.solver = solver
        self.month = None
        self.load(month, clim)

    def load(self, month: int, clim: dict | None = None) -> None:
        """Band tables of `month` (1..12) on the device (rad_load_aerosols; at start-up and month changes)."""
        import ctypes

        from . import _lib
        c, keep = _clim_struct(clim if clim is not None else climatology(month))
        s = self.solver
        _lib.check(s.lib, s.handle, s.lib.rad_load_aerosols(s.handle, ctypes.byref(c)), "rad_load_aerosols")
        self.month = month

    def optics(self, dev: dict, rhly, xlon, xlat, slmsk, out: tuple | None = None, stream=None,
               ivflip: int = 0) -> tuple:
        """faersw [3, 14, nlay, ncol], faerlw [3, 16, nlay, ncol] (CUDA float32) for the columns of `dev` (the
        tensors of RadSolver.to_device: plvl, plyr, tlyr, qlyr) and the CUDA tensors rhly [nlay, ncol], xlon,
        xlat, slmsk [ncol] (radians, mask 0 / 1 / 2).  ivflip 1: the layers of the inputs and of the outputs are
        surface first (the reference's other orientation; its ivflip = 1 statements mirror the top-first ones,
        so the top-first kernel runs on the reversed layers, through temporary tensors)."""
        import ctypes

        import torch

        from . import _lib
        if ivflip not in (0, 1):
            raise ValueError("aerosol optics: ivflip must be 0 or 1")
        if ivflip == 1:
            st = stream if stream is not None else torch.cuda.current_stream()
            with torch.cuda.stream(st):
                rev = {k: torch.flip(dev[k], dims=[0]).contiguous() for k in ("plvl", "plyr", "tlyr", "qlyr")}
                top = self.optics(rev, torch.flip(rhly, dims=[0]).contiguous(), xlon, xlat, slmsk, stream=st)
                if out is None:
                    out = tuple(torch.empty_like(t) for t in top)
                for o, t in zip(out, top):
                    if tuple(o.shape) != tuple(t.shape):
                        raise ValueError(f"aerosol optics: out must be {tuple(t.shape)}")
                    o.copy_(torch.flip(t, dims=[2]))
            return out
        nlay, ncol = dev["plyr"].shape
        if nlay != self.solver.cfg.nlay:
            raise ValueError(f"aerosol optics: the columns have {nlay} layers, the solver {self.solver.cfg.nlay}")
        a = _lib.RadAerColumns()
        src = {"plvl": dev["plvl"], "plyr": dev["plyr"], "tlyr": dev["tlyr"], "qlyr": dev["qlyr"], "rhly": rhly,
               "xlon": xlon, "xlat": xlat, "slmsk": slmsk}
        shapes = {"plvl": (nlay + 1, ncol), "xlon": (ncol,), "xlat": (ncol,), "slmsk": (ncol,)}
        for k, v in src.items():
            if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float32 and v.is_contiguous()):
                raise TypeError(f"aerosol input {k} must be a contiguous float32 CUDA tensor")
            if tuple(v.shape) != shapes.get(k, (nlay, ncol)):
                raise ValueError(f"aerosol input {k} has shape {tuple(v.shape)}, expected {shapes.get(k, (nlay, ncol))}")
            setattr(a, k, v.data_ptr())
        if out is None:
            out = (torch.empty((3, 14, nlay, ncol), dtype=torch.float32, device=dev["plyr"].device),
                   torch.empty((3, 16, nlay, ncol), dtype=torch.float32, device=dev["plyr"].device))
        for o, nb in zip(out, (14, 16)):
            if not (isinstance(o, torch.Tensor) and o.is_cuda and o.dtype == torch.float32 and o.is_contiguous()
                    and tuple(o.shape) == (3, nb, nlay, ncol)):
                raise ValueError(f"aerosol optics: out must be contiguous float32 CUDA tensors [3, {nb}, {nlay}, {ncol}]")
        st = stream if stream is not None else torch.cuda.current_stream()
        s = self.solver
        rc = s.lib.rad_setaer(s.handle, ctypes.byref(a), ncol, ctypes.c_void_p(out[0].data_ptr()),
                              ctypes.c_void_p(out[1].data_ptr()), ctypes.c_void_p(st.cuda_stream))
        _lib.check(s.lib, s.handle, rc, "rad_setaer")
        return out


def volcanic(solver, plvl, xlat, ivolae, kyrsav: int, kmonsav: int, faer: tuple, ivflip: int = 0,
             add_sw: bool = True, add_lw: bool = True, lw1bd: bool = False, stream=None) -> tuple:
    """setaer's stratospheric volcanic term (lavoflg; rad_setaer_volc) added in place to the extinction of
    faer = (faersw [3, 14, nlay, ncol], faerlw [3, 16, nlay, ncol]) CUDA float32, after Aerosols.optics.
    plvl [nlay + 1, ncol] mb in the order of ivflip and xlat [ncol] radians: contiguous float32 CUDA tensors;
    ivolae: the int32 [10, 4, 12] (year, zone, month) table on the host (numpy or a CPU tensor), read for year
    kyrsav mod 10 and month kmonsav."""
    import ctypes

    import numpy as np
    import torch

    from . import _lib
    for k, v in (("plvl", plvl), ("xlat", xlat), ("faersw", faer[0]), ("faerlw", faer[1])):
        if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float32 and v.is_contiguous()):
            raise TypeError(f"volcanic input {k} must be a contiguous float32 CUDA tensor")
    iv = ivolae.cpu().numpy() if isinstance(ivolae, torch.Tensor) else ivolae
    iv = np.ascontiguousarray(iv, dtype=np.int32)
    if iv.shape != (10, 4, 12):
        raise ValueError(f"ivolae must be int32 [10, 4, 12], got {iv.shape}")
    nlay, ncol = solver.cfg.nlay, plvl.shape[1]
    if (tuple(plvl.shape) != (nlay + 1, ncol) or tuple(xlat.shape) != (ncol,)
            or tuple(faer[0].shape) != (3, 14, nlay, ncol) or tuple(faer[1].shape) != (3, 16, nlay, ncol)):
        raise ValueError(f"volcanic: expected plvl [{nlay + 1}, ncol], xlat [ncol], faersw [3, 14, {nlay}, ncol] and "
                         f"faerlw [3, 16, {nlay}, ncol] (the solver's {nlay} layers)")
    st = stream if stream is not None else torch.cuda.current_stream()
    s = solver
    rc = s.lib.rad_setaer_volc(s.handle, ctypes.c_void_p(plvl.data_ptr()), ctypes.c_void_p(xlat.data_ptr()), ncol,
                               int(ivflip), iv.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), int(kyrsav),
                               int(kmonsav), int(bool(add_sw)), int(bool(add_lw)), int(bool(lw1bd)),
                               ctypes.c_void_p(faer[0].data_ptr()), ctypes.c_void_p(faer[1].data_ptr()),
                               ctypes.c_void_p(st.cuda_stream))
    _lib.check(s.lib, s.handle, rc, "rad_setaer_volc")
    return faer
