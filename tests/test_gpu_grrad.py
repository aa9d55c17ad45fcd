"""grrad's radiation-layer set-up on the GPU (rad_grrad_setup through the C-ABI) against the golden vectors
of the reference's kernels and against the oracle on 65,536 columns; the radiation solved on the GPU's layers
against the float64 oracle solved on the oracle's.  CUDA's powf / expf / logf differ from the host's in the
last bits, so values agree to relative 2e-6 (pressures, temperatures and the copied fields bit for bit),
saturation and relative humidity to 2e-5 (the saturation pressure interpolates between two closed-form
powf / expf nodes)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import assert_within
from oracle import oracle
from woof_nam_b200.columns import Columns, make_columns, model_state

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "grrad_golden.npz"
EXACT = ("plvl", "plyr", "tlyr", "qlyr", "tsfg")


def _gpu(m):
    import torch
    from woof_nam_b200.grrad import layers
    from woof_nam_b200.solver import RadSolver
    s = RadSolver()
    out = layers(s, {k: torch.as_tensor(np.ascontiguousarray(v), device="cuda") for k, v in m.items()})
    torch.cuda.synchronize()
    return s, out


def _check(out, ref, what):
    for k in oracle.GRRAD_FIELDS:
        g = out[k].cpu().numpy()
        assert g.shape == ref[k].shape, (what, k)
        if k in EXACT:
            assert np.array_equal(g, ref[k]), (what, k)
        else:
            e = np.abs(g.astype(np.float64) - ref[k]) / np.maximum(np.abs(ref[k]), 1e-12)
            assert e.max() < (2e-5 if k in ("rhly", "qstl") else 2e-6), (what, k, e.max())


@pytest.mark.parametrize("case", ["plain", "stress"])
def test_golden(case):
    z = np.load(GOLDEN)
    m = {k: z[f"{case}_in_{k}"] for k in ("pint", "pmid", "prslk", "t", "q", "tsfc")}
    _, out = _gpu(m)
    _check(out, {k: z[f"{case}_{k}"] for k in oracle.GRRAD_FIELDS}, case)


def test_layers_feed_the_solve():
    cols = make_columns(65536, 321)
    m = model_state(cols)
    ref_lay = oracle.grrad_setup(m)
    s, lay = _gpu(m)
    _check(lay, ref_lay, "65536 columns")
    # the columns as grrad builds them: its layers, the request's gases, clouds and surface
    kw = {f: getattr(cols, f) for f in Columns.FIELDS}
    kw.update({k: ref_lay[k] for k in ("plvl", "plyr", "tlyr", "tlvl", "qlyr")}, tsfg=ref_lay["tsfg"])
    built = Columns(**kw)
    sub = built.slice(0, 2048)
    ref = oracle.solve(sub, precision="double")
    dev = s.to_device(sub)
    for k in ("plvl", "plyr", "tlyr", "tlvl", "qlyr"):
        dev[k] = lay[k][:, :2048].contiguous()
    dev["tsfg"] = lay["tsfg"][:2048].contiguous()
    out = s.solve(dev, sub.solcon)
    assert_within({k: v.cpu().numpy().astype(np.float64) for k, v in out.items()}, ref, what="solve on grrad's layers")
