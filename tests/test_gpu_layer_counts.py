"""Requests with other layer counts than the parent grid's 61: the top 21 layers dropped (40 layers, the model
top at 216 hPa) and the three lowest layers split in two (64 layers, NLAY_MAX).  The gas-optics task tiling,
the per-layer set-up and the sweeps all index by the request's nlay, so the mixed kernels must stay within the
tolerances (0.05 W/m^2, 0.01 K/day), on the tiled path and on the single-kernel forms, and the float64
kernels close to the float64 oracle: 2e-3 W/m^2 and 2e-3 K/day, as in the float64 stress test (on these 2,048
columns the float64 kernel's SW heating differs from the oracle's by up to 1.0e-3 K/day in all three layer
counts, the unmodified 61 included, so the difference belongs to the columns and not to the layer count)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_within
from oracle import oracle
from woof_nam_b200.columns import Columns, make_columns

pytestmark = pytest.mark.gpu


def with_layers(cols: Columns, nlay: int) -> Columns:
    """cols (61 layers, top first) with the top layers dropped (nlay < 61) or the lowest layers split in two at
    their mid-pressure (nlay > 61): a split layer's halves keep its temperature, humidity, gases and cloud fraction
    and sizes and take half its cloud paths each."""
    f = {k: np.asarray(getattr(cols, k), np.float64) for k in Columns.FIELDS}
    n0 = cols.nlay
    if nlay <= n0:
        m = n0 - nlay
        for k in ("plyr", "tlyr", "qlyr", "olyr"):
            f[k] = f[k][m:]
        for k in ("plvl", "tlvl"):
            f[k] = f[k][m:]
        for k in ("gasvmr", "clouds"):
            f[k] = f[k][:, m:]
    else:
        for j in range(n0 - 1, n0 - 1 - (nlay - n0), -1):      # the lowest layers, bottom up
            pm = 0.5 * (f["plvl"][j] + f["plvl"][j + 1])
            f["plvl"] = np.insert(f["plvl"], j + 1, pm, axis=0)
            f["tlvl"] = np.insert(f["tlvl"], j + 1, f["tlyr"][j], axis=0)
            for k in ("tlyr", "qlyr", "olyr"):
                f[k] = np.insert(f[k], j + 1, f[k][j], axis=0)
            for k in ("gasvmr", "clouds"):
                f[k] = np.insert(f[k], j + 1, f[k][:, j], axis=1)
            f["clouds"][1, j:j + 2] *= 0.5
            f["clouds"][3, j:j + 2] *= 0.5
            f["plyr"] = np.insert(f["plyr"], j + 1, 0.0, axis=0)
            f["plyr"][j] = 0.5 * (f["plvl"][j] + f["plvl"][j + 1])
            f["plyr"][j + 1] = 0.5 * (f["plvl"][j + 1] + f["plvl"][j + 2])
    kw = {k: np.ascontiguousarray(v, np.float32) for k, v in f.items()}
    out = Columns(**kw, solcon=cols.solcon, diagnostic_clouds=cols.diagnostic_clouds)
    assert out.nlay == nlay and out.plvl.shape[0] == nlay + 1
    assert (np.diff(out.plvl.astype(np.float64), axis=0) > 0).all()
    return out


@pytest.fixture(scope="module", params=[40, 61, 64])
def request_of(request):
    cols = with_layers(make_columns(2048, 4242), request.param)
    return cols, oracle.solve(cols, precision="double")


@pytest.mark.parametrize("form", ["tiled", "single"])
def test_mixed_other_layer_counts(request_of, form):
    from woof_nam_b200.solver import RadSolver
    cols, ref = request_of
    kw = dict(lw_chunk=-1, sw_sweep_chunk=-1) if form == "single" else {}
    out = RadSolver(precision="mixed", nlay=cols.nlay, **kw).solve_host(cols)
    assert_within(out, ref, what=f"mixed kernels, {cols.nlay} layers, {form}")


def test_fp64_other_layer_counts(request_of):
    from woof_nam_b200.solver import RadSolver
    cols, ref = request_of
    out = RadSolver(precision="fp64", nlay=cols.nlay).solve_host(cols)
    e = assert_within(out, ref, flux_tol=2e-3, heat_tol=2e-3, what=f"fp64 kernel, {cols.nlay} layers")
    print(cols.nlay, {k: f"{v:.2e}" for k, v in e.items()})
