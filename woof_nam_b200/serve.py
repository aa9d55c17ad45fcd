"""Continuous-batching radiation server on one GPU.

Requests are radiation solves of whole domains (the 12 km parent, the 3 km nests) for ensemble members,
arriving over time.  The server

  * keeps each member's column state resident on the device (uploaded once, refreshed in place),
  * admits a request when its output buffers fit the HBM budget beside the resident state and the slots'
    library scratch (held per slot from start-up) and a stream slot is free, so requests that arrive while
    others run start at once and overlap on the device,
  * runs every admitted solve on its own CUDA stream and library handle (a handle's scratch is not shared
    between concurrent solves), tracks completion with CUDA events,
  * reports latency from arrival to completion (p50 / p99) and throughput in columns/s.

Each result depends only on its own request (the SW MINVAL(laytrop) groups are request-local and the
kernels reduce in a fixed order), so a request gives the same bits alone and in the mix.

    python -m woof_nam_b200.serve --requests 40 --rate 40 --members 10
"""
from __future__ import annotations

import argparse
import json
import time
from dataclasses import dataclass, field

import numpy as np

from .columns import make_columns
from .solver import RadSolver, output_shapes

DOMAINS = {"180x180": 180 * 180, "333x333": 333 * 333, "600x450": 600 * 450, "954x835": 954 * 835}


@dataclass
class Request:
    rid: int
    domain: str
    member: int
    arrival: float                 # seconds after the server start
    start: float = -1.0
    done: float = -1.0
    ncol: int = 0
    out: dict | None = None         # outputs, kept when the server runs with keep_outputs

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class _Slot:
    solver: RadSolver
    stream: object
    req: Request | None = None
    event: object = None
    out: dict = field(default_factory=dict)


class RadServer:
    """members[domain] -> list of device-resident column dicts (one per member)."""

    def __init__(self, states: dict, solcon: float, slots: int = 4, hbm_budget_gb: float = 120.0,
                 precision: str = "mixed", keep_outputs: bool = False, policy: str = "fifo"):
        """policy: the order in which queued requests take free slots -- "fifo" (arrival order) or "sjf" (the
        request with the fewest columns first, arrival order among equals)."""
        import torch
        if policy not in ("fifo", "sjf"):
            raise ValueError(f"RadServer: policy must be 'fifo' or 'sjf', got {policy!r}")
        self.policy = policy
        self.torch = torch
        self.states = states
        self.solcon = solcon
        self.budget = int(hbm_budget_gb * 1e9)
        self.resident = sum(t.numel() * t.element_size() for dom in states.values() for m in dom for t in m.values())
        if self.resident > self.budget:
            raise MemoryError(f"resident column state {self.resident / 1e9:.1f} GB exceeds the HBM budget")
        from .solver import SolverConfig
        from .tune import tuned_config
        largest = max(int(m["coszen"].shape[-1]) for dom in states.values() for m in dom)
        # launch shape for the largest domain, LW chunks of at most 32,768 columns (3.1 GB of scratch a slot),
        # SW chunks of 8,192 day columns (3.2 GB a slot)
        cfg = tuned_config(largest, SolverConfig(precision=precision, sw_sweep_chunk=8192), max_chunk=32768)
        self.slots = [_Slot(RadSolver(cfg), torch.cuda.Stream()) for _ in range(slots)]
        # each slot's handle keeps the scratch it grows to (up to the largest request) until it is closed
        self.held = sum(sl.solver.workspace_bytes(largest) for sl in self.slots)
        if self.resident + self.held > self.budget:
            raise MemoryError(f"resident state {self.resident / 1e9:.1f} GB and slot scratch "
                              f"{self.held / 1e9:.1f} GB exceed the HBM budget")
        self.in_use = 0
        self.keep = keep_outputs

    def request_bytes(self, ncol: int, solver: RadSolver) -> int:
        """Device bytes a request adds while it is in flight: its output arrays (the slot's scratch is held
        already and counted at start-up)."""
        return sum(int(np.prod(s)) * 4 for s in output_shapes(solver.cfg.nlay, ncol).values())

    def _ncol(self, req: Request) -> int:
        return int(self.states[req.domain][req.member]["coszen"].shape[-1])

    def _launch(self, slot: _Slot, req: Request, now: float):
        torch = self.torch
        cols = self.states[req.domain][req.member]
        req.ncol = int(cols["coszen"].shape[-1])
        with torch.cuda.stream(slot.stream):
            slot.out = slot.solver.alloc_outputs(req.ncol)
            slot.solver.solve(cols, self.solcon, slot.out, stream=slot.stream)
            slot.event = torch.cuda.Event()
            slot.event.record(slot.stream)
        slot.req = req
        req.start = now

    def run(self, requests: list, poll_s: float = 2e-4) -> dict:
        """Serve requests (sorted by arrival); returns per-request timings and the summary."""
        torch = self.torch
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: list = []
        done: list = []
        t0 = time.perf_counter()
        nreq = len(pending)
        while len(done) < nreq:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            for sl in self.slots:                      # completions
                if sl.req is not None and sl.event.query():
                    sl.req.done = time.perf_counter() - t0
                    done.append(sl.req)
                    self.in_use -= self.request_bytes(sl.req.ncol, sl.solver)
                    if self.keep:
                        sl.req.out = sl.out
                    sl.req, sl.out = None, {}
            for sl in self.slots:                      # admissions: a free slot and room in the budget
                if sl.req is None and queue:
                    qi = 0
                    if self.policy == "sjf":
                        qi = min(range(len(queue)), key=lambda i: (self._ncol(queue[i]), queue[i].arrival))
                    r = queue[qi]
                    need = self.request_bytes(self._ncol(r), sl.solver)
                    if self.resident + self.held + self.in_use + need > self.budget:
                        break
                    queue.pop(qi)
                    self.in_use += need
                    self._launch(sl, r, time.perf_counter() - t0)
            if pending and not queue and all(sl.req is None for sl in self.slots):
                time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.01)))
            else:
                time.sleep(poll_s)
        torch.cuda.synchronize()
        wall = max(r.done for r in done) - min(r.arrival for r in done)
        lat = np.array([r.latency for r in done]) * 1e3
        cols = sum(r.ncol for r in done)
        return {"requests": nreq, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "columns": cols, "wall_s": wall, "columns_per_s": cols / wall,
                "slots": len(self.slots), "resident_gb": self.resident / 1e9, "slot_scratch_gb": self.held / 1e9,
                "lw_chunk": self.slots[0].solver.cfg.lw_chunk}


def poisson_requests(n: int, rate: float, members: int, seed: int = 7) -> list:
    """n requests with exponential inter-arrival times (mean 1/rate s), domains drawn uniformly from the
    parent and nest sizes, members uniformly from 0..members-1."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    names = list(DOMAINS)
    return [Request(i, names[rng.integers(len(names))], int(rng.integers(members)), float(t[i])) for i in range(n)]


def member_states(members: int, device: str = "cuda", seed: int = 3030, sizes: dict | None = None) -> dict:
    """Device-resident column states: one seeded state per domain size, and per member a copy perturbed on
    the device (temperature +- 1 K, humidity x (1 +- 5 %), member-specific) so members differ."""
    import torch
    from .solver import RadSolver as _RS
    sizes = sizes or DOMAINS
    out = {}
    gen = torch.Generator(device=device)
    for i, (name, n) in enumerate(sizes.items()):
        base = make_columns(n, seed + i)
        d0 = _RS.to_device(None, base, device=device)
        out[name] = []
        for m in range(members):
            gen.manual_seed(seed * 131 + i * 17 + m)
            d = {k: v.clone() for k, v in d0.items()}
            d["tlyr"] += (torch.rand(d["tlyr"].shape, generator=gen, device=device) - 0.5) * 2.0
            d["qlyr"] *= 1.0 + (torch.rand(d["qlyr"].shape, generator=gen, device=device) - 0.5) * 0.1
            out[name].append(d)
        del d0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=40)
    ap.add_argument("--rate", type=float, default=40.0)
    ap.add_argument("--members", type=int, default=10)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    args = ap.parse_args()
    import torch
    from .columns import SOLCON
    states = member_states(args.members)
    torch.cuda.synchronize()
    srv = RadServer(states, SOLCON, slots=args.slots, hbm_budget_gb=args.budget_gb)
    warm = [Request(-1, name, 0, 0.0) for name in DOMAINS]
    srv.run(warm)
    res = srv.run(poisson_requests(args.requests, args.rate, args.members))
    res.update({"rate_per_s": args.rate, "members": args.members, "budget_gb": args.budget_gb})
    print(json.dumps(res))


if __name__ == "__main__":
    main()
