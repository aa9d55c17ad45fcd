"""rad_solve_noalloc (fixed scratch array, no allocator) against rad_solve through the C ABI: two calls in
a row give rad_solve's outputs (on a handle with the single-kernel LW and SW, lw_chunk < 0 and
sw_sweep_chunk < 0, the forms the no-allocation entry runs), and requests the fixed region cannot hold are
refused before any launch.
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
    s = RadSolver(precision=precision, lw_chunk=-1, sw_sweep_chunk=-1)
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
    s = RadSolver(precision="mixed", route="mcica", lw_chunk=-1, sw_sweep_chunk=-1)
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


def test_noalloc_fresh_handle_allocates_nothing():
    """A handle that has never solved: rad_solve_noalloc leaves the device's free memory unchanged (no
    scratch is created for it), twice in a row, and its outputs agree with rad_solve's within the mixed
    path's tolerance (0.05 W/m^2, 0.01 K/day: rad_solve runs the two-kernel LW here, the entry the single-
    kernel LW)."""
    import torch
    from conftest import assert_within
    from woof_nam_b200.solver import RadSolver
    warm = RadSolver(precision="mixed")                 # the library's first use on the device happens here
    c = make_columns(512, 45)
    rc, _ = _call(warm, warm.to_device(c), c.solcon, None, torch.cuda.current_stream())
    assert rc == 0, warm.lib.rad_last_error(warm.handle)
    s = RadSolver(precision="mixed")
    st = torch.cuda.current_stream()
    for n, seed in ((4000, 46), (2500, 47)):
        c = make_columns(n, seed)
        d = s.to_device(c)
        out = s.alloc_outputs(n)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc, got = _call(s, d, c.solcon, out, st)
        assert rc == 0, s.lib.rad_last_error(s.handle)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, "rad_solve_noalloc changed the device's free memory"
        got = {k: v.cpu().numpy() for k, v in got.items()}
        ref = s.solve_host(c)
        assert_within(got, ref, what="rad_solve_noalloc vs rad_solve")


def test_noalloc_refuses_above_max():
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver(precision="mixed")
    c = make_columns(MAX_COLS + 1, 44)
    d = s.to_device(c)
    rc, _ = _call(s, d, c.solcon, None, torch.cuda.current_stream())
    assert rc == _lib.RAD_E_INVALID and b"RAD_NOALLOC_MAX_COLS" in s.lib.rad_last_error(s.handle)
