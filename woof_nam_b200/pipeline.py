"""Solves of host-resident requests with the host<->device copies overlapped (double buffering).

A model that keeps its state on the host hands the radiation call its columns every step and reads the outputs
back.  Done one after the other, the 4.9 GB of inputs of the 954 x 835 parent grid cost ~90 ms of PCIe per step on
top of the solve.  Here each request goes to one of `depth` device buffer sets: its host->device copy runs on one
copy stream while the previous request solves on the compute stream, and its device->host copy on a second copy
stream while the next one solves, so a step costs max(solve, copy) instead of their sum:

    h2d stream:  H2D(i)      H2D(i+1)            H2D(i+2)  (waits for solve(i): same buffers)
    compute:            solve(i)      solve(i+1)           (waits for H2D(i); for D2H(i-depth): same outputs)
    d2h stream:                  D2H(i)        D2H(i+1)    (waits for solve(i))

    from woof_nam_b200.pipeline import HostPipeline
    pipe = HostPipeline(solver, ncol)
    for step in range(n):
        pipe.submit(host_inputs[step], solcon, host_outputs[step])   # pinned host tensors; returns at once
    pipe.synchronize()

Host buffers must be pinned (page-locked) for the copies to be asynchronous, and a request's host inputs and
outputs must stay untouched until `done(i)` (or `synchronize()`).  Results are the same bits as `solver.solve`
on the same inputs (tests/test_gpu_pipeline.py).
"""
from __future__ import annotations

from .solver import INPUT_FIELDS


class HostPipeline:
    def __init__(self, solver, ncol: int, depth: int = 2, device="cuda", inputs=INPUT_FIELDS):
        import torch
        if depth < 2:
            raise ValueError("HostPipeline: depth must be at least 2 to overlap copies with solves")
        self.torch = torch
        self.device = torch.device(device)
        self.solver = solver
        self.ncol = int(ncol)
        self.depth = depth
        self.inputs = tuple(inputs)
        self.h2d, self.comp, self.d2h = torch.cuda.Stream(device), torch.cuda.Stream(device), torch.cuda.Stream(device)
        self.din = [None] * depth
        self.dout = [solver.alloc_outputs(self.ncol, device=device) for _ in range(depth)]
        self.solved = [None] * depth      # solve of the request in the slot done (its inputs free, outputs ready)
        self.drained = [None] * depth     # D2H of the request in the slot done (its outputs free)
        self.events = {}                  # request -> its D2H-done event (completed ones pruned)
        self.n = 0

    def _inputs_like(self, hin: dict) -> dict:
        torch = self.torch
        return {k: torch.empty(v.shape, dtype=v.dtype, device=self.device) for k, v in hin.items()}

    def submit(self, hin: dict, solcon: float, hout: dict) -> int:
        """Queue request n: hin / hout map the solve's input / output names to pinned host tensors.  Returns n."""
        torch = self.torch
        s = self.n % self.depth
        if self.din[s] is None:
            self.din[s] = self._inputs_like(hin)
        din, dout = self.din[s], self.dout[s]
        with torch.cuda.stream(self.h2d):
            if self.solved[s] is not None:
                self.h2d.wait_event(self.solved[s])          # the slot's previous solve has read its inputs
            for k, v in hin.items():
                din[k].copy_(v, non_blocking=True)
            copied = torch.cuda.Event()
            copied.record(self.h2d)
        self.comp.wait_event(copied)
        if self.drained[s] is not None:
            self.comp.wait_event(self.drained[s])            # the slot's previous outputs have been read back
        self.solver.solve(din, solcon, dout, stream=self.comp)
        solved = torch.cuda.Event()
        solved.record(self.comp)
        self.solved[s] = solved
        with torch.cuda.stream(self.d2h):
            self.d2h.wait_event(solved)
            for k, v in hout.items():
                v.copy_(dout[k], non_blocking=True)
            drained = torch.cuda.Event()
            drained.record(self.d2h)
        self.drained[s] = drained
        self.events[self.n] = drained
        # the D2H copies complete in order, so a completed event stands for every request before it: keep a few
        while len(self.events) > 4 * self.depth:
            i0 = min(self.events)
            if not self.events[i0].query():
                break
            del self.events[i0]
        self.n += 1
        return self.n - 1

    def done(self, i: int) -> bool:
        """True once request i's outputs are in its host buffers."""
        if not 0 <= i < self.n:
            raise ValueError(f"HostPipeline: request {i} was never submitted")
        ev = self.events.get(i)
        return True if ev is None else ev.query()      # pruned events had completed

    def wait_on(self, stream) -> None:
        """Make `stream` wait for every request submitted so far (their outputs on the host)."""
        if self.events:
            stream.wait_event(self.events[max(self.events)])

    def start_after(self, stream) -> None:
        """Make the pipeline's streams wait for the work queued on `stream` so far (e.g. a timing event)."""
        torch = self.torch
        ev = torch.cuda.Event()
        ev.record(stream)
        for st in (self.h2d, self.comp, self.d2h):
            st.wait_event(ev)

    def synchronize(self) -> None:
        for st in (self.h2d, self.comp, self.d2h):
            st.synchronize()
