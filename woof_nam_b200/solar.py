"""Solar geometry of a radiation call: the sun at the forecast time (rad_sol_update, host) and the mean
cosine of the solar zenith angle of every column over the SW interval (rad_coszmn, device).

    from woof_nam_b200.solar import sol_update, coszmn
    sun = sol_update((2026, 7, 1, 12, 0, 0), deltsw=1200.0, deltim=25.0)   # NAM: NRADS 48 x 25 s
    coszen, coszdg = coszmn(solver, sun, glon, glat, solhr=12.0, dtswav=1200.0 / 3600.0, nrads=48)

coszen (the daytime mean) is the SW's SW_COSZEN input and day predicate (>= 1e-4); coszdg (the mean over
the whole interval) is the post step's COSZDG_V; sun["solcon"] is the solar constant at the day's sun-earth
distance.
"""
from __future__ import annotations

import ctypes

from . import _lib

SOLC0 = 1366.0     # solar constant at 1 AU without a yearly table, W/m^2


def sol_update(date, deltsw: float, deltim: float, solc0: float = SOLC0) -> dict:
    """sollag, sindec, cosdec, anginc, solcon, nstp at date = (year, month, day, hour, minute, second)."""
    lib = _lib.load()
    a = _lib.RadSolarIn(*[int(x) for x in date], float(deltsw), float(deltim), float(solc0))
    s = _lib.RadSolarState()
    rc = lib.rad_sol_update(ctypes.byref(a), ctypes.byref(s))
    if rc != 0:
        raise ValueError(lib.rad_last_error(None).decode())
    out = {k: getattr(s, k) for k, _ in s._fields_}
    out["_state"] = s
    return out


def coszmn(solver, sun: dict, glon, glat, solhr: float, dtswav: float, nrads: int, out=None, stream=None):
    """(coszen, coszdg) CUDA float32 tensors shaped like glon for CUDA float32 glon / glat (radians)."""
    import torch
    for name, t in (("glon", glon), ("glat", glat)):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
            raise TypeError(f"coszmn: {name} must be a contiguous float32 CUDA tensor")
    if glat.shape != glon.shape:
        raise ValueError(f"coszmn: glat {tuple(glat.shape)} and glon {tuple(glon.shape)} differ")
    if out is None:
        out = (torch.empty_like(glon), torch.empty_like(glon))
    for name, t in zip(("coszen", "coszdg"), out):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and t.shape == glon.shape):
            raise ValueError(f"coszmn: out {name} must be a contiguous float32 CUDA tensor shaped like glon")
    st = stream if stream is not None else torch.cuda.current_stream()
    rc = solver.lib.rad_coszmn(solver.handle, ctypes.byref(sun["_state"]), ctypes.c_void_p(glon.data_ptr()),
                               ctypes.c_void_p(glat.data_ptr()), glon.numel(), float(solhr), float(dtswav), int(nrads),
                               ctypes.c_void_p(out[0].data_ptr()), ctypes.c_void_p(out[1].data_ptr()),
                               ctypes.c_void_p(st.cuda_stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_coszmn")
    return out
