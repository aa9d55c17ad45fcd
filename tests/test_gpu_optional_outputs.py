"""lwrad's and swrad's optional outputs through the C-ABI against the float64 oracle: clear-sky heating
(hlw0, HSW0), heating per band (hlwb 16 bands, HTSWB 14 bands) and level-flux profiles (flwprf, FLXPRF) --
the fields the reference's units write when lhlw0 / lhlwb / lhsw0 / lhswb (has_htrswb) / lflxprf are on
(phys_rrtm_lw_lwrad.py:47-50, phys_rrtm_sw_swrad.py:49-51).  Heating within 0.01 K/day per band and in
total, fluxes within 0.05 W/m^2; the main outputs stay what a solve without them gives."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import FLUX_TOL, HEAT_TOL, assert_within
from oracle import oracle
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu

ALL = dict(lhsw0=True, lhswb=True, lhlw0=True, lhlwb=True, lflxprf=True)
HEAT = ("hsw0", "htswb", "hlw0", "hlwb")
FLUX = ("swflxprf", "lwflxprf")


def _check(out, ref, what):
    for k in HEAT:
        d = np.abs(out[k].astype(np.float64) - ref[k]) * 86400.0
        assert d.max() <= HEAT_TOL, f"{what} {k}: {d.max():.3e} K/day (band maxima {d.reshape(-1, d.shape[-2] * d.shape[-1]).max(axis=1) if d.ndim == 3 else ''})"
    for k in FLUX:
        d = np.abs(out[k].astype(np.float64) - ref[k])
        assert d.max() <= FLUX_TOL, f"{what} {k}: {d.max():.3e} W/m^2"


@pytest.mark.parametrize("seed,stress", [(1001, False), (5005, True)])
def test_optional_outputs_against_oracle(seed, stress):
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(4096 if not stress else 2048, seed, stress=stress)
    ref = oracle.solve(cols, precision="double", diag=True)
    out = RadSolver(precision="mixed", diagnostic=stress, **ALL).solve_host(cols)
    _check(out, ref, f"seed {seed}")
    assert_within(out, ref, what="main outputs beside the optional ones")
    plain = RadSolver(precision="mixed", diagnostic=stress).solve_host(cols)
    for k in plain:
        assert np.array_equal(plain[k], out[k]), k
    # the bands add up to the total-sky heating as the reference's do
    assert np.abs(out["htswb"].astype(np.float64).sum(0) - out["htsw"]).max() * 86400.0 < 2e-3
    assert np.abs(out["hlwb"].astype(np.float64).sum(0) - out["htlw"]).max() * 86400.0 < 2e-3


def test_night_columns_and_parts():
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(300, 7)
    cols.coszen[:150] = -0.3
    out = RadSolver(precision="mixed", **ALL).solve_host(cols)
    for k in ("hsw0", "htswb", "swflxprf"):
        assert (out[k][..., :150] == 0).all(), k
    ref = oracle.solve(cols, precision="double", diag=True)
    _check(out, ref, "half night")
    lw = RadSolver(precision="mixed", parts="lw", lhlw0=True, lhlwb=True, lflxprf=True).solve_host(cols)
    assert "hsw0" not in lw and np.abs(lw["hlw0"] - out["hlw0"]).max() == 0


def test_refused_where_not_produced():
    import torch
    from woof_nam_b200._lib import RAD_E_INVALID, RadError
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(64, 8)
    with pytest.raises(RadError):
        RadSolver(precision="mixed", lw_chunk=-1, lhlw0=True).solve_host(cols)
    with pytest.raises(RadError):
        RadSolver(precision="fp64", lhsw0=True).solve_host(cols)
    s = RadSolver(precision="mixed", lhswb=True)
    d = s.to_device(cols)
    ci, co, n, _ = s._abi_args(d, cols.solcon, None)
    rc = s.lib.rad_solve_noalloc(s.handle, ctypes.byref(ci), ctypes.byref(co), n,
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == RAD_E_INVALID and b"optional outputs" in s.lib.rad_last_error(s.handle)
