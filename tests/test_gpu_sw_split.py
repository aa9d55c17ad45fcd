"""The two-kernel SW (sw4_optics_kernel + sw4_sweep_kernel: set-up, optics and the layer R/T of a chunk of day
columns into the chunk scratch, then the adding sweeps from it) against the single-kernel SW (sw_sweep_chunk
< 0) through the C-ABI, with chunks smaller than the day count (several chunks, a ragged last one, chunks past
the day count that exit at once), with aerosol optics, on the McICA route, and against the float64 oracle
within the mixed-precision tolerances (0.05 W/m^2, 0.01 K/day).  Both forms run the same statements and make
the same float64 / table-entry decisions; the compiler may fuse a multiply and an add differently in the two
kernels, so the outputs agree to float rounding (relative 1e-5 of each output's scale), not to the bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_within
from oracle import oracle
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu


def _solve(cols, chunk, faersw=None, **kw):
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver(precision="mixed", parts="sw", sw_sweep_chunk=chunk, **kw)
    dev = s.to_device(cols)
    if faersw is not None:
        dev["faersw"] = faersw
    out = s.solve(dev, cols.solcon)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _aerosol(ncol, nlay=61, seed=12):
    """Band optical depth, single-scattering albedo and asymmetry [3 x 14][nlay][ncol] of plausible size."""
    import torch
    g = torch.Generator().manual_seed(seed)
    tau = torch.rand(14, nlay, ncol, generator=g) * 0.2
    ssa = 0.8 + 0.19 * torch.rand(14, nlay, ncol, generator=g)
    asy = 0.5 + 0.3 * torch.rand(14, nlay, ncol, generator=g)
    return torch.cat([tau, ssa, asy]).contiguous().cuda()


def _equal(a, b, what):
    for k in a:
        scale = max(float(np.abs(b[k]).max()), 1e-30)
        d = float(np.abs(a[k].astype(np.float64) - b[k]).max())
        assert d <= 1e-5 * scale, f"{what}: {k} differs by {d:.3e} (scale {scale:.3e})"


@pytest.mark.parametrize("chunk", [0, 333, 512])
def test_split_equals_single_kernel(chunk):
    cols = make_columns(3000, 4711)
    _equal(_solve(cols, chunk), _solve(cols, -1), f"sw_sweep_chunk {chunk}")


def test_split_with_aerosol():
    cols = make_columns(2500, 4712)
    fsw = _aerosol(cols.ncol)
    _equal(_solve(cols, 700, fsw), _solve(cols, -1, fsw), "aerosol")


def test_split_mcica():
    cols = make_columns(2000, 4713)
    _equal(_solve(cols, 256, route="mcica"), _solve(cols, -1, route="mcica"), "mcica")


def test_split_against_oracle():
    cols = make_columns(2048, 4714)
    ref = oracle.solve(cols, precision="double")
    out = _solve(cols, 300)
    assert_within(out, {k: ref[k] for k in out}, what="two-kernel SW")
