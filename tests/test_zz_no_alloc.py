"""rad_solve_noalloc (fixed scratch array, no allocator) against rad_solve through the C ABI: two calls in
a row give rad_solve's outputs (on a handle with the single-kernel LW, lw_chunk < 0, the form the
no-allocation entry runs), and requests the fixed region cannot hold are refused before any launch.
The file name sorts last so the test also runs after every other GPU test of the session."""
from __future__ import annotations

import ctypes

import pytest

from woof_nam_b200 import _lib
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu

MAX_COLS = 65536


def _call(s, cols, solcon, out, stream):
    ci, co, ncol, out = s._abi_args(cols, solcon, out)
    return s.lib.rad_solve_noalloc(s.handle, ctypes.byref(ci), ctypes.byref(co), ncol,
                                   ctypes.c_void_p(stream.cuda_stream)), out


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_noalloc_equals_solve_twice(precision):
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver(precision=precision, lw_chunk=-1)
    st = torch.cuda.current_stream()
    for n, seed in ((3001, 41), (777, 42)):           # two calls in a row, the second smaller
        c = make_columns(n, seed)
        d = s.to_device(c)
        ref = s.solve(d, c.solcon)
        rc, got = _call(s, d, c.solcon, None, st)
        assert rc == 0, s.lib.rad_last_error(s.handle)
        torch.cuda.synchronize()
        for k, v in ref.items():
            # the same arithmetic on the same inputs (the SW here recomputes its layer R/T where rad_solve
            # reads them back from its store): equal to the bit, far inside the 0.05 W/m^2 / 0.01 K/day
            # tolerance of the mixed path
            assert torch.equal(v, got[k]), (precision, n, k)


def test_noalloc_mcica_with_caller_masks():
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver(precision="mixed", route="mcica", lw_chunk=-1)
    c = make_columns(1500, 43)
    d = s.to_device(c)
    ref = s.solve(d, c.solcon)
    st = torch.cuda.current_stream()
    rc, got = _call(s, d, c.solcon, s.alloc_outputs(1500), st)
    assert rc == 0, s.lib.rad_last_error(s.handle)
    torch.cuda.synchronize()
    for k, v in ref.items():
        assert torch.equal(v, got[k]), k
    out = s.alloc_outputs(1500)
    del out["lw_mask"]
    rc, _ = _call(s, d, c.solcon, out, st)
    assert rc == _lib.RAD_E_INVALID and b"lw_mask" in s.lib.rad_last_error(s.handle)


def test_noalloc_refuses_above_max():
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver(precision="mixed")
    c = make_columns(MAX_COLS + 1, 44)
    d = s.to_device(c)
    rc, _ = _call(s, d, c.solcon, None, torch.cuda.current_stream())
    assert rc == _lib.RAD_E_INVALID and b"RAD_NOALLOC_MAX_COLS" in s.lib.rad_last_error(s.handle)
