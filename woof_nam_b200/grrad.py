"""grrad's radiation layers from the model state on the GPU (rad_grrad_setup): the set-up and layer part of
the NMMB radiation driver ahead of the column solve.

    from woof_nam_b200.grrad import layers
    lay = layers(solver, model)     # model: CUDA tensors pint [lm + 1, n], pmid, prslk, t, q [lm, n], tsfc [n]
    dev.update({k: lay[k] for k in ("plvl", "plyr", "tlyr", "tlvl", "qlyr", "tsfg")})   # RadColumns fields

lm model layers give lm + 1 radiation layers (the extra top layer); pressures in Pa in, mb out.  rhly is
the aerosol optics' humidity, qstl / prslk1 / tvly the cloud and ozone set-up's inputs.
"""
from __future__ import annotations

import ctypes

from . import _lib


def layers(solver, model: dict, out: dict | None = None, stream=None) -> dict:
    import torch
    for k in _lib.MODEL_FIELDS:
        v = model[k]
        if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float32 and v.is_contiguous()):
            raise TypeError(f"grrad layers: {k} must be a contiguous float32 CUDA tensor")
    lm, n = model["pmid"].shape
    dev = model["pmid"].device
    inshape = {"pint": (lm + 1, n), "tsfc": (n,)}
    for k in _lib.MODEL_FIELDS:
        if tuple(model[k].shape) != inshape.get(k, (lm, n)):
            raise ValueError(f"grrad layers: {k} has shape {tuple(model[k].shape)}, expected {inshape.get(k, (lm, n))}")
    shapes = {"plvl": (lm + 2, n), "tlvl": (lm + 2, n), "tsfg": (n,)}
    if out is None:
        out = {k: torch.empty(shapes.get(k, (lm + 1, n)), dtype=torch.float32, device=dev) for k in _lib.LAYER_FIELDS}
    for k in _lib.LAYER_FIELDS:
        v = out[k]
        if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float32 and v.is_contiguous()
                and tuple(v.shape) == shapes.get(k, (lm + 1, n))):
            raise ValueError(f"grrad layers: out {k} must be a contiguous float32 CUDA tensor {shapes.get(k, (lm + 1, n))}")
    a, o = _lib.RadModelColumns(), _lib.RadLayerFields()
    for k in _lib.MODEL_FIELDS:
        setattr(a, k, model[k].data_ptr())
    for k in _lib.LAYER_FIELDS:
        setattr(o, k, out[k].data_ptr())
    st = stream if stream is not None else torch.cuda.current_stream()
    rc = solver.lib.rad_grrad_setup(solver.handle, ctypes.byref(a), n, lm, ctypes.byref(o), ctypes.c_void_p(st.cuda_stream))
    _lib.check(solver.lib, solver.handle, rc, "rad_grrad_setup")
    return out
