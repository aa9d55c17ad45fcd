"""McICA route on the GPU: sub-column cloud words bit-exact against the oracle (which is pinned to the
reference's generators), fluxes and heating rates within the tolerances of the float64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_within
from oracle import oracle
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu


def _solver(**kw):
    from woof_nam_b200.solver import RadSolver
    return RadSolver(route="mcica", precision="mixed", **kw)


@pytest.mark.parametrize("iovr", [0, 1, 2])
def test_masks_bit_exact(iovr):
    cols = make_columns(700, 31)
    ref = oracle.mcica_masks(cols, iovrlw=iovr, iovrsw=iovr)
    out = _solver(iovrlw=iovr, iovrsw=iovr).solve_host(cols)
    assert np.array_equal(out["lw_mask"], ref["lw"])
    assert np.array_equal(out["sw_mask"], ref["sw"])


def test_masks_explicit_seeds():
    cols = make_columns(300, 32)
    seeds = np.random.default_rng(5).integers(-2**31, 2**31 - 1, size=(2, cols.ncol)).astype(np.int32)
    ref = oracle.mcica_masks(cols, icseed=seeds)
    out = _solver().solve_host(cols, icseed=seeds)
    assert np.array_equal(out["lw_mask"], ref["lw"])
    assert np.array_equal(out["sw_mask"], ref["sw"])


def test_mcica_fluxes_within_tolerance():
    cols = make_columns(1024, 33)
    ref = oracle.solve(cols, precision="double", route=1)
    out = _solver().solve_host(cols)
    assert_within(out, ref, what="McICA route, plain request")


def test_mcica_stress_within_tolerance():
    cols = make_columns(512, 34, stress=True)
    ref = oracle.solve(cols, precision="double", route=1)
    out = _solver(diagnostic=True).solve_host(cols)
    assert_within(out, ref, what="McICA route, precision-stress request")
