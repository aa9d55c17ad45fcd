"""Argument checks that need no GPU: the serving engine refuses an unknown admission policy, and the solver refuses
inputs whose sizes disagree with its layer count or the request's columns before any library call."""
from __future__ import annotations

import pytest


def test_unknown_policy_refused():
    pytest.importorskip("torch")
    from woof_nam_b200.serve import RadServer
    with pytest.raises(ValueError, match="policy"):
        RadServer({}, 1368.22, policy="lifo")


def _stub(nlay=61, parts="both"):
    from woof_nam_b200.solver import RadSolver, SolverConfig
    s = object.__new__(RadSolver)          # the argument checks only; no device handle
    s.cfg = SolverConfig(nlay=nlay, parts=parts)
    return s


def _cols(nlay=61, ncol=8):
    import torch
    from woof_nam_b200.solver import input_shapes
    return {k: torch.zeros(v) for k, v in input_shapes(nlay, ncol).items() if k not in ("faerlw", "faersw", "icseed")}


def test_solver_refuses_mis_sized_inputs_before_the_library():
    """Every input is checked against the solver's layer count and the request's columns (the kernels index by
    those alone), before the device check; layout-equivalent shapes ([42][nlay][ncol] for faersw) pass."""
    torch = pytest.importorskip("torch")
    s = _stub()
    for k, bad in (("gasvmr", (10, 60, 8)), ("plvl", (61, 8)), ("sfcalb", (3, 8)), ("clouds", (9, 61, 7))):
        c = _cols()
        c[k] = torch.zeros(bad)
        with pytest.raises(ValueError, match=k):
            s._abi_args(c, 1368.22, None)
    c = _cols()
    c["faersw"] = torch.zeros(42, 61, 8)
    with pytest.raises(TypeError):       # shapes pass; host tensors are refused next
        s._abi_args(c, 1368.22, None)
    c["faersw"] = torch.zeros(42, 60, 8)
    with pytest.raises(ValueError, match="faersw"):
        s._abi_args(c, 1368.22, None)
    with pytest.raises(ValueError, match="layers"):
        _stub(nlay=40)._abi_args(_cols(), 1368.22, None)
