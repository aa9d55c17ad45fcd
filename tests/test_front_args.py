"""The front-end wrappers refuse host tensors and mis-shaped arrays before they reach the library: the kernels
index by the sizes passed beside the pointers, so a host pointer or a short array would be read or written out
of bounds on the device.  No GPU needed (the checks run before any library call)."""
from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")

from woof_nam_b200 import _lib, front  # noqa: E402

N, NLAY = 8, 5


def _z(*shape, dtype=None):
    return torch.zeros(shape, dtype=dtype or torch.float32)


def test_host_tensors_refused():
    with pytest.raises(TypeError):
        front.dayparts(None, _z(N), _z(N), _z(N), 12.0, 1.0, 4, {}, im=4)
    with pytest.raises(TypeError):
        front.getgases(None, _z(NLAY + 1, N), _z(N), _z(N), co2_glb=_z(1), gco2cyc=_z(12),
                       co2vmr_sav=_z(12, 12, 24), ico2flg=2, kmonsav=7, ivflip=0)
    with pytest.raises(TypeError):
        front.getozn(None, _z(NLAY, N), _z(N), o3r=_z(12, 4, 18), pkstr=_z(4), k1oz=1, k2oz=2, facoz=0.5,
                     blte=-85.0, dlte=10.0)
    with pytest.raises(TypeError):
        front.setalb(None, {k: _z(N) for k in _lib.ALBEDO_FIELDS}, 1)
    with pytest.raises(TypeError):
        front.setemis(None, {k: _z(N) for k in _lib.EMIS_FIELDS[:-1]}, None, 1, 0)
    with pytest.raises(TypeError):
        front.progcld2(None, {k: _z(NLAY + 1 if k == "plvl" else NLAY, N) for k in _lib.CLOUD_IN_FIELDS[:-1]},
                       ivflip=0, llyr=2, iovr=1)


def test_mis_shaped_outputs_refused():
    with pytest.raises(ValueError):
        front.getgases(None, _z(NLAY + 1, N), _z(N), _z(N), gasvmr=_z(10, NLAY, N + 1), co2_glb=None,
                       gco2cyc=None, co2vmr_sav=None, ico2flg=0, kmonsav=None, ivflip=0)
