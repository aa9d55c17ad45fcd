"""The C-ABI serving queue (rad_queue_create / rad_submit / rad_poll / rad_wait): requests submitted while
others run start at once on free slots, every ticket's outputs equal rad_solve's on the same handle, and the
queue answers BUSY, BUDGET, INVALID and TIMEOUT as documented."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from woof_nam_b200 import _lib
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu


def _queue(solvers, budget=0):
    lib = solvers[0].lib
    hs = (ctypes.c_void_p * len(solvers))(*[s.handle.value for s in solvers])
    q = ctypes.c_void_p()
    assert lib.rad_queue_create(hs, len(solvers), budget, ctypes.byref(q)) == 0, lib.rad_last_error(None)
    return lib, q


def test_submitted_requests_overlap_and_equal_solve():
    import torch
    from woof_nam_b200.solver import RadSolver
    slots = [RadSolver(precision="mixed") for _ in range(3)]
    lib, q = _queue(slots)
    reqs = [make_columns(n, 900 + n) for n in (5000, 1234, 20000, 700, 3333)]
    dev = [slots[0].to_device(c) for c in reqs]
    outs, tickets, pending = [None] * len(reqs), [0] * len(reqs), list(range(len(reqs)))
    busy_seen = False
    while pending or any(t > 0 for t in tickets):
        while pending:
            i = pending[0]
            ci, co, n, o = slots[0]._abi_args(dev[i], reqs[i].solcon, None)
            t = ctypes.c_int64()
            rc = lib.rad_submit(q, ctypes.byref(ci), ctypes.byref(co), n, ctypes.byref(t))
            if rc == _lib.RAD_E_BUSY:
                busy_seen = True
                break
            assert rc == 0, lib.rad_last_error(None)
            outs[i], tickets[i] = o, t.value
            pending.pop(0)
        for i, t in enumerate(tickets):
            if t > 0:
                done = ctypes.c_int32()
                assert lib.rad_poll(q, t, ctypes.byref(done)) == 0
                if done.value:
                    tickets[i] = -t
    assert busy_seen                                   # 5 requests, 3 slots
    lib.rad_queue_destroy(q)
    torch.cuda.synchronize()
    ref = RadSolver(precision="mixed")
    for c, o in zip(reqs, outs):
        r = ref.solve_host(c)
        for k, v in r.items():
            assert np.array_equal(v, o[k].cpu().numpy()), k


def test_budget_timeout_and_unknown_ticket():
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver(precision="mixed")
    small, big = make_columns(512, 1), make_columns(40000, 2)
    need_big = s.workspace_bytes(40000)
    s2 = RadSolver(precision="mixed")              # the queue does not own its slot handles: keep them alive
    lib, q = _queue([s, s2], budget=need_big + s.workspace_bytes(512) // 2)
    d = s.to_device(big)
    ci, co, n, o = s._abi_args(d, big.solcon, None)
    t = ctypes.c_int64()
    assert lib.rad_submit(q, ctypes.byref(ci), ctypes.byref(co), n, ctypes.byref(t)) == 0, lib.rad_last_error(None)
    ds = s.to_device(small)
    ci2, co2, n2, _ = s._abi_args(ds, small.solcon, None)
    t2 = ctypes.c_int64()
    rc = lib.rad_submit(q, ctypes.byref(ci2), ctypes.byref(co2), n2, ctypes.byref(t2))
    assert rc == _lib.RAD_E_BUDGET, (rc, lib.rad_last_error(None))
    rc = lib.rad_wait(q, t.value, 0)
    assert rc in (0, _lib.RAD_E_TIMEOUT)
    assert lib.rad_wait(q, t.value, 60000) == 0
    assert lib.rad_submit(q, ctypes.byref(ci2), ctypes.byref(co2), n2, ctypes.byref(t2)) == 0
    assert lib.rad_wait(q, t2.value, 60000) == 0
    done = ctypes.c_int32()
    assert lib.rad_poll(q, 999, ctypes.byref(done)) == _lib.RAD_E_INVALID
    assert lib.rad_poll(q, t.value, ctypes.byref(done)) == 0 and done.value == 1
    lib.rad_queue_destroy(q)
    torch.cuda.synchronize()
    del s2
