"""Benchmark of the RRTM LW+SW column radiation: columns/s on the 12 km NAM parent grid (954 x 835 columns,
60 model layers = 61 radiation layers), mixed-precision CUDA path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one LW+SW solve of the whole domain (796,590 columns) with inputs resident in HBM.  Under
torchrun (N > 1) every rank solves its own ensemble member of the same size (weak scaling; columns are
independent, so there is no data-path collective); the time is the max over ranks.  Rank 0 prints one
JSON line.  The reference arm (--impl reference) times the reference's own RRTM kernels compiled for the
host CPU (oracle/_ref) on a bounded sample of the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "c2_parent_954x835"
METRIC = "LW+SW columns/s at 60 levels"
UNIT = "columns/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
TRAFFIC = ROOT / "profiles" / "traffic.json"
B200_SMS, FP32_LANES_PER_SM = 148, 128
CPU_SAMPLE = 16384


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 kernel leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the uneven-batch leg (parent grid + three nests in one graph-captured launch set)")
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE)
    ap.add_argument("--no-aer", action="store_true", help="skip the aerosol-optics leg")
    ap.add_argument("--no-front", action="store_true", help="skip the grrad front-end leg")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity block (errors against the oracle)")
    ap.add_argument("--parity-sample", type=int, default=16384)
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--lw-chunk", type=int, default=None,
                    help="LW chunk size (columns); default: the autotuner's choice for this device")
    ap.add_argument("--sw-chunk", type=int, default=None,
                    help="SW tile of sunlit columns; default: the autotuner's choice (with --lw-chunk: 16384)")
    ap.add_argument("--ncol", type=int, default=None,
                    help="solve this many columns of the workload's generator instead of the full domain "
                         "(small cases for profiling)")
    return ap.parse_args()


def peaks():
    try:
        return json.loads(PEAKS.read_text())
    except (OSError, ValueError):
        return {}


def fp32_peak_tflops(pk):
    """FP32 FMA pipe: 148 SMs x 128 lanes x 2 FLOP x the measured max SM clock."""
    mhz = float(pk.get("sm_max_mhz", 1965.0))
    return B200_SMS * FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12, mhz


# ---------------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap,pci.bus_id")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus = (bus_id or "").lower()
        self.rows, self.proc, self.th = [], None, None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.th:
                self.th.join(timeout=5)
        rows = [r for r in self.rows if len(r) >= 8]
        mine = [r for r in rows if self.bus and self.bus.endswith(r[7].lower()[-12:])] or rows
        if not mine:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in mine if r[0].replace(".", "").isdigit()]
        reasons = sorted({self.REASONS[i] for r in mine for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(mine[0][1]) if mine[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(mine)}


# ---------------------------------------------------------------------------------------------------
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return ws, int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle
    from woof_nam_b200.columns import workload
    which = "ref" if oracle.REF_LIB.exists() else "port"
    cols = workload(args.workload, ncol=args.cpu_sample)
    nth = oracle.host_threads()
    for _ in range(max(args.warmup, 0)):
        oracle.solve(cols, precision="float", which=which, nthreads=nth)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.solve(cols, precision="float", which=which, nthreads=nth)
    dt = (time.perf_counter() - t0) / args.steps
    v = cols.ncol / dt
    sample = (f"{cols.ncol} columns of the {args.workload} generator per step (FP32 reference kernels, "
              f"LW on every column, SW on the {int((cols.coszen >= 1e-4).sum())} sunlit ones)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "columns_per_step": cols.ncol, "layers": cols.nlay},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "kind": "reference" if which == "ref" else "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def cpu_baseline(cols, n_sample):
    from oracle import oracle
    which = "ref" if oracle.REF_LIB.exists() else "port"
    sub = cols.slice(0, min(n_sample, cols.ncol))
    nth = oracle.host_threads()
    oracle.solve(sub.slice(0, 256), precision="float", which=which, nthreads=nth)
    t0 = time.perf_counter()
    oracle.solve(sub, precision="float", which=which, nthreads=nth)
    dt = time.perf_counter() - t0
    return {"value": sub.ncol / dt, "unit": UNIT, "cores": nth, "kind": "reference" if which == "ref" else "port",
            "sample": f"first {sub.ncol} columns of the timed workload, one solve, FP32 "
                      f"{'reference kernels compiled for the host' if which == 'ref' else 'oracle restatement'}, "
                      f"{dt:.1f} s"}


def parity_block(cols, mcfg, n_sample):
    """Errors of the timed path against the float64 oracle on the first n_sample columns of the timed workload,
    through the same solver configuration with lwrad's / swrad's optional outputs on: the largest absolute error
    of every output (heating K/day, fluxes W/m^2), of every band's heating (hlwb 16 LW bands, htswb 14 SW bands),
    and the count of values above the tolerances (0.01 K/day, 0.05 W/m^2)."""
    from oracle import oracle
    from woof_nam_b200.solver import RadSolver, SolverConfig
    sub = cols.slice(0, min(n_sample, cols.ncol))
    flags = dict(lhsw0=True, lhswb=True, lhlw0=True, lhlwb=True, lflxprf=True)
    s = RadSolver(SolverConfig(**{**mcfg.__dict__, **flags}))
    got = s.solve_host(sub)
    s.close()
    ref = oracle.solve(sub, precision="double", diag=True, nthreads=oracle.host_threads())
    heat = ("htlw", "htsw", "hlw0", "hsw0", "hlwb", "htswb")
    flux = ("topflw", "sfcflw", "topfsw", "sfcfsw", "fdncmp", "lwflxprf", "swflxprf")

    def err(k):
        o, r = np.asarray(got[k], np.float64), np.asarray(ref[k], np.float64)
        d = np.where(np.isfinite(o) & np.isfinite(r), np.abs(o - r), np.inf)
        return d * (86400.0 if k in heat else 1.0)

    e = {k: err(k) for k in heat + flux}
    return {
        "sample": f"first {sub.ncol} columns of the timed workload ({int((sub.coszen >= 1e-4).sum())} sunlit), "
                  f"float64 oracle (C++ restatement of the reference statements)",
        "tolerance": {"heating_K_per_day": 0.01, "flux_W_per_m2": 0.05},
        "max_abs": {k: float(v.max()) for k, v in e.items() if k not in ("hlwb", "htswb")},
        "max_abs_per_band": {"hlwb": [float(x) for x in e["hlwb"].reshape(16, -1).max(axis=1)],
                             "htswb": [float(x) for x in e["htswb"].reshape(14, -1).max(axis=1)]},
        "values_over_tolerance": {k: int((v > (0.01 if k in heat else 0.05)).sum()) for k, v in e.items()},
        "values": int(sum(v.size for v in e.values())),
    }


def serving_block(members: int, n_req: int, seed: int = 7) -> dict:
    """The serving workload (Poisson arrivals of whole-domain solves drawn from the parent grid and the three
    nests, ensemble members resident on the device, admission by a 120 GB HBM budget, 4 slots): once at the
    configured 40 requests/s, which offers ~12 M columns/s (beyond what one GPU serves, so latency there is
    queueing), and once at 80 % of the rate the GPU sustained in that run, where the queue stays short.  Latency
    from arrival to completion; offered and served columns/s."""
    from woof_nam_b200 import serve
    from woof_nam_b200.columns import SOLCON
    states = serve.member_states(members)
    srv = serve.RadServer(states, SOLCON, slots=4, hbm_budget_gb=120.0)
    srv.run([serve.Request(-1, name, 0, 0.0) for name in serve.DOMAINS])
    mean_cols = float(np.mean(list(serve.DOMAINS.values())))

    def leg(rate, s):
        r = srv.run(serve.poisson_requests(n_req, rate, members, seed=s))
        return {"rate_per_s": rate, "offered_columns_per_s": rate * mean_cols, "served_columns_per_s": r["columns_per_s"],
                "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "mean_ms": r["mean_ms"], "requests": r["requests"]}

    sat = leg(40.0, seed)
    sus_rate = 0.8 * sat["served_columns_per_s"] / mean_cols
    sus = leg(sus_rate, seed + 1)
    res = {"workload": f"Poisson arrivals, domains uniform over {list(serve.DOMAINS)} x 61 layers, {members} members "
                       f"resident ({srv.resident / 1e9:.1f} GB), HBM budget 120 GB, 4 slots "
                       f"({srv.held / 1e9:.1f} GB of slot scratch), admission in arrival order",
           "at_40_per_s": sat, "sustainable": sus}
    # the same two arrival sequences with the fewest-columns-first admission
    del srv
    srv = serve.RadServer(states, SOLCON, slots=4, hbm_budget_gb=120.0, policy="sjf")
    srv.run([serve.Request(-1, name, 0, 0.0) for name in serve.DOMAINS])
    res["shortest_first"] = {"at_40_per_s": leg(40.0, seed), "sustainable": leg(sus_rate, seed + 1)}
    del srv, states
    return res


def front_block(mixed, cols, dev, seed: int, tstep, steps: int, warmup: int, im: int = 954) -> dict:
    """grrad's front end for the timed domain: each front-end kernel alone (HBM roofline: the algorithmic bytes
    of a column -- every input word read once, every output word written once -- times the columns, over the
    kernel's CUDA-event time), then the whole radiation call (chain.radiation_call: the front end feeding the
    solve, one stream) per step.  The NAM settings: ico2flg 1, ntoz 0 climatological ozone, Ferrier clouds
    (np3d 3, ivflip 0), ialbflg 2 (and the MODIS branch 1 for comparison), iemslw 1.  Inputs: the columns'
    model state (model_state), seeded surface fields and climatologies (columns.surface_state, front_tables)
    and cloud fields (cloud_state of a 65,536-column tile repeated across the domain), on a NAM-like grid
    (-140..-60 E, 10..60 N)."""
    import torch
    from woof_nam_b200 import front, solar
    from woof_nam_b200.chain import CLOUD_NAM, radiation_call
    from woof_nam_b200.columns import cloud_state, front_tables, model_state, surface_state
    from woof_nam_b200.grrad import layers as grrad_layers
    n = cols.ncol
    jm = n // im
    T = lambda a, dt=None: torch.as_tensor(np.ascontiguousarray(a, dtype=dt), device=dev)  # noqa: E731
    model = {k: T(v) for k, v in model_state(cols).items()}
    lm = model["pmid"].shape[0]
    lmk = lm + 1
    lay = grrad_layers(mixed, model)
    tile = min(n, 65536)
    lay_t = {k: v[..., :tile].cpu().numpy() for k, v in lay.items()}
    cld_t = cloud_state(lay_t, seed)
    reps = -(-n // tile)
    cld = {k: T(np.tile(cld_t[k], (1, reps))[:, :n] if cld_t[k].ndim == 2 else np.tile(cld_t[k], reps)[:n])
           for k in ("clw", "f_ice", "f_rain", "r_rime", "cldfk1")}
    sfc_h = surface_state(n, seed + 1)
    lon = np.deg2rad(np.linspace(-140.0, -60.0, im))[None, :].repeat(jm, 0).ravel()
    lat = np.deg2rad(np.linspace(10.0, 60.0, jm))[:, None].repeat(im, 1).ravel()
    sfc_h.update(glon=lon, glat=lat, sinlat=np.sin(lat), coslat=np.cos(lat))
    sfc = {k: T(v, np.float32) for k, v in sfc_h.items()}
    tab_h = front_tables(seed + 2)
    tab = {k: (T(v) if isinstance(v, np.ndarray) else v) for k, v in tab_h.items()}
    tab["co2_glb"] = T(np.atleast_1d(np.float32(tab_h["co2_glb"])))
    # 12:40 UTC: the morning terminator crosses the middle of the grid, so about half of it is sunlit (as the
    # solve's columns are) and the call's SW work compares with the solve's
    sun = solar.sol_update((2026, 7, 1, 12, 40, 0), deltsw=1200.0, deltim=25.0)
    call = dict(solhr=12.0 + 40.0 / 60.0, dtswav=1200.0 / 3600.0, nrads=48)
    f32 = dict(dtype=torch.float32, device=dev)
    gas, oz = torch.empty((10, lmk, n), **f32), torch.zeros((lmk, n), **f32)
    alb, ems = torch.empty((4, n), **f32), torch.empty(n, **f32)
    dp = front.dayparts(mixed, sfc["glon"], sfc["sinlat"], sfc["coslat"], sun=sun, im=im, **call)
    sfc["coszf"] = dp["coszen"]
    cin = {k: lay[k] for k in ("plyr", "plvl", "tlyr", "tvly", "qlyr", "qstl", "rhly")}
    cin.update(cld, xlat=sfc["glat"])
    cl = front.progcld2(mixed, cin, **CLOUD_NAM)
    # the cloud tracers grrad sums into clw (NAM: one, the condensate, at ntcw 2) and the surface albedo the
    # IALB = 2 block starts from
    tracer = torch.stack([cld["clw"] * 0.5, cld["clw"], cld["clw"] * 0.25]).contiguous()
    clw = torch.empty_like(cld["clw"])
    sfc["sfcalbedo"] = sfc["alvsf"].clone()
    pay = front.payne_albedo(mixed, sfc["sfcalbedo"], sfc["sm"], dp["coszen"])
    run = {
        "k_grrad_setup": (lambda: grrad_layers(mixed, model, out=lay), 4 * (14 * lm + 14)),
        "k_dayparts": (lambda: front.dayparts(mixed, sfc["glon"], sfc["sinlat"], sfc["coslat"], sun=sun, im=im, out=dp,
                                              **call), 20),
        "k_getozn": (lambda: front.getozn(mixed, lay["prslk1"], sfc["glat"], oz, o3r=tab["o3r"], pkstr=tab["pkstr"],
                                          k1oz=6, k2oz=7, facoz=0.4, blte=tab["blte"], dlte=tab["dlte"]),
                     4 * (2 * lmk + 1)),
        "k_getgases": (lambda: front.getgases(mixed, lay["plvl"], sfc["glon"], sfc["glat"], gas, co2_glb=tab["co2_glb"],
                                              gco2cyc=tab["gco2cyc"], co2vmr_sav=tab["co2vmr_sav"], ico2flg=1,
                                              kmonsav=7, ivflip=0), 4 * 10 * lmk),
        "k_grrad_clw": (lambda: front.grrad_clw(mixed, tracer, 2, 1, clw=clw), 4 * 2 * lmk),
        "k_progcld2": (lambda: front.progcld2(mixed, cin, out=cl, **CLOUD_NAM), 4 * (8 * lmk + 2 + 9 * lmk + 11)),
        "k_payne_albedo": (lambda: front.payne_albedo(mixed, sfc["sfcalbedo"], sfc["sm"], dp["coszen"], out=pay),
                           4 * (3 + 9)),
        "k_setalb(ialbflg 2)": (lambda: front.setalb(mixed, sfc, 2, alb), 32),
        "k_setalb(ialbflg 1)": (lambda: front.setalb(mixed, sfc, 1, alb), 4 * (16 + 4)),
        "k_setemis": (lambda: front.setemis(mixed, sfc, tab["idxems"], 2, 1, ems), 4 * (9 + 1)),
    }
    hbm = float(peaks().get("hbm_gbs", 6650.0))
    kern = {}
    for name, (fn, bpc) in run.items():
        ms = tstep(fn, steps, warmup)
        gbs = bpc * n / (ms * 1e-3) / 1e9
        kern[name] = {"ms": ms, "bytes_per_column": bpc, "achieved_gbs": gbs, "frac": gbs / hbm}
    state = dict(model)
    state.update(cld)
    state.update(sfc)
    state["tracer1"] = tracer
    clim = dict(tab)
    kw = dict(sun=sun, im=im, kmonsav=7, k1oz=6, k2oz=7, facoz=0.4, ico2flg=1, ialbflg=2, iemslw=1, ntcw=2, **call)
    first = radiation_call(mixed, state, clim, **kw)
    work, outs = first["work"], {k: v for k, v in first.items() if k != "work"}
    ms_call = tstep(lambda: radiation_call(mixed, state, clim, work=work, out=outs, **kw), steps, warmup)
    front_ms = sum(v["ms"] for k, v in kern.items() if k != "k_setalb(ialbflg 1)")
    nday = int((dp["coszen"] >= 1e-4).sum().item())
    res = {"workload": f"{im}x{jm} columns x {lmk} layers, NAM settings (ico2flg 1, climatological ozone, Ferrier "
                       f"clouds, ialbflg 2, iemslw 1); seeded surface / cloud / climatology stand-ins",
           "kernels": kern, "front_end_ms": front_ms, "peak_gbs": hbm,
           "radiation_call": {"value": n / (ms_call * 1e-3), "unit": UNIT, "ms_per_step": ms_call, "day_columns": nday,
                              "what": "chain.radiation_call: grrad set-up, dayparts, getozn, getgases, clw from the "
                                      "cloud tracers, progcld2, the IALB = 2 albedo, setalb, setemis and the LW+SW "
                                      "solve of the whole domain, one stream, no row windows"}}
    del state, clim, work, outs, first, model, lay, cld, sfc, tab, tracer, clw, pay
    return res


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    from oracle import oracle
    from woof_nam_b200.columns import WORKLOADS, workload, make_columns
    from woof_nam_b200.solver import RadSolver, INPUT_FIELDS

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if ws > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n, seed, stress = WORKLOADS[args.workload]
    n = args.ncol or n
    # weak scaling: rank r solves ensemble member r (same generator, seed offset by the rank)
    cols = make_columns(n, seed + 7919 * rank, stress)
    nday = int((cols.coszen >= np.float32(1e-4)).sum())
    # launch shape (LW chunk) from the autotuner, measured outside the timed region and cached per device
    from woof_nam_b200.solver import SolverConfig
    from woof_nam_b200.tune import tuned_config
    mcfg = SolverConfig(precision="mixed", diagnostic=stress)
    if args.lw_chunk is None and args.sw_chunk is None:
        mcfg = tuned_config(n, mcfg)
    else:
        mcfg = SolverConfig(**{**mcfg.__dict__, "lw_chunk": args.lw_chunk or 32768, "sw_sweep_chunk": args.sw_chunk or 0})
    mixed = RadSolver(mcfg)
    d = mixed.to_device(cols, device=dev)
    out = mixed.alloc_outputs(n, device=dev)
    in_bytes = sum(d[k].numel() * 4 for k in INPUT_FIELDS)
    out_bytes = sum(v.numel() * 4 for v in out.values())
    stream = torch.cuda.current_stream()

    def timed(solver, steps, warmup, profile=False, sampler=None):
        for _ in range(warmup):
            solver.solve(d, cols.solcon, out)
        torch.cuda.synchronize()
        barrier()
        if profile:
            solver.profile(True)
        launches0 = solver.profile_read()["launches"]
        if sampler:
            sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            solver.solve(d, cols.solcon, out)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps)
        prof = solver.profile_read()
        if profile:
            solver.profile(False)
        return ms, prof, prof["launches"] - launches0, clocks

    def tstep(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    bus = None
    try:
        p = torch.cuda.get_device_properties(dev)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    except Exception:
        pass
    ms, prof, launches, clocks = timed(mixed, args.steps, args.warmup, profile=True, sampler=ClockSampler(bus))
    value = ws * n / (ms * 1e-3)

    # plain FP64 single-domain kernel (the reference statements in FP64): the x8 denominator
    fp64 = None
    if not args.no_fp64:
        s64 = RadSolver(precision="fp64", diagnostic=stress)
        ms64, _, _, _ = timed(s64, max(1, min(args.steps, 3)), max(args.warmup, 1))
        fp64 = {"value": ws * n / (ms64 * 1e-3), "ms_per_step": ms64, "unit": UNIT}
        del s64

    # end to end through the public API with host buffers: pinned host inputs -> device, solve, -> host
    hin = {k: v.cpu().pin_memory() for k, v in d.items()}
    hout = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in out.items()}

    def e2e_step():
        for k in INPUT_FIELDS:
            d[k].copy_(hin[k], non_blocking=True)
        mixed.solve(d, cols.solcon, out)
        for k, v in out.items():
            hout[k].copy_(v, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    # the same, double-buffered through the public HostPipeline: each step's host->device copy overlaps the previous
    # step's solve and its device->host copy the next one's (two device buffer sets, three streams)
    from woof_nam_b200.pipeline import HostPipeline
    pipe = HostPipeline(mixed, n, depth=2, device=dev)
    for _ in range(args.warmup):
        pipe.submit(hin, cols.solcon, hout)
    pipe.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pipe.start_after(stream)
    for _ in range(args.steps):
        pipe.submit(hin, cols.solcon, hout)
    pipe.wait_on(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_pipe = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    del pipe

    # uneven batch: the parent grid plus the 3 km nests (333x333, 600x450, 180x180) as one batched solve
    # captured in a CUDA graph, replayed per step; the nests' inputs are resident too
    batch = None
    if not args.no_batch and args.ncol is None:
        from woof_nam_b200.columns import NESTS
        nest_cols = [make_columns(jm * im, seed + 101 * (i + 1) + 7919 * rank, stress) for i, (jm, im) in enumerate(NESTS)]
        reqs = [d] + [mixed.to_device(c, device=dev) for c in nest_cols]
        graph = mixed.capture(reqs, [cols.solcon] + [c.solcon for c in nest_cols])
        for _ in range(args.warmup):
            graph.launch(stream)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            graph.launch(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_b = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        nb = n + sum(c.ncol for c in nest_cols)
        batch = {"value": ws * nb / (ms_b * 1e-3), "unit": UNIT, "ms_per_step": ms_b, "columns": nb,
                 "requests": 1 + len(nest_cols), "graph": True,
                 "workload": "954x835 parent + 333x333, 600x450, 180x180 nests, one batched launch set per step"}
        graph.close()
        del reqs, graph

    # climatological aerosol optics (setaer / aer_property, NAM iaer = 11) of the same columns: the kernel alone
    # (HBM roofline: 5 nlay + 4 input words and 90 nlay output words per column), then the radiation step with
    # aerosol (optics + the solve reading them)
    aer = None
    if not args.no_aer:
        from woof_nam_b200 import aerosols
        A = aerosols.Aerosols(mixed, month=1)
        ai = {k: torch.as_tensor(np.ascontiguousarray(v), device=dev)
              for k, v in aerosols.make_inputs(cols, seed + rank, "nam").items()}
        da = dict(d)
        da["faersw"], da["faerlw"] = A.optics(d, ai["rhly"], ai["xlon"], ai["xlat"], ai["slmsk"])
        opt = lambda: A.optics(d, ai["rhly"], ai["xlon"], ai["xlat"], ai["slmsk"], out=(da["faersw"], da["faerlw"]))  # noqa: E731

        ms_a = tstep(opt, args.steps, args.warmup)
        ms_as = tstep(lambda: (opt(), mixed.solve(da, cols.solcon, out)), args.steps, args.warmup)
        nl = cols.nlay
        bpc = 4 * ((5 * nl + 1 + 3) + 3 * 30 * nl)
        hbm = float(peaks().get("hbm_gbs", 6650.0))
        aer = {"kernel": "k_setaer", "month": 1, "ms": ms_a, "columns_per_s": ws * n / (ms_a * 1e-3),
               "bytes_per_column": bpc, "achieved_gbs": bpc * n / (ms_a * 1e-3) / 1e9, "peak_gbs": hbm,
               "frac": bpc * n / (ms_a * 1e-3) / 1e9 / hbm,
               "step_with_aerosol": {"value": ws * n / (ms_as * 1e-3), "unit": UNIT, "ms_per_step": ms_as}}
        del da, A

    # grrad's front end of the same domain and the whole radiation call (front end + solve)
    front_leg = None
    if not args.no_front and args.ncol is None:
        front_leg = front_block(mixed, cols, dev, seed + rank, tstep, args.steps, args.warmup)

    # roofline of the dominant kernel (FP32 pipe; algorithmic FLOPs from the oracle's operation-count table)
    pk = peaks()
    peak_tf, mhz = fp32_peak_tflops(pk)
    ops = oracle.opcount(cols.slice(0, 1024))
    lw_ms, sw_ms = prof["lw_ms"] / max(prof["solves"], 1), prof["sw_ms"] / max(prof["solves"], 1)
    lw_tf = ops["lw_flops_per_col"] * n / (lw_ms * 1e-3) / 1e12
    sw_tf = ops["sw_flops_per_daycol"] * nday / (sw_ms * 1e-3) / 1e12
    # the mixed precision runs the two-kernel LW (gas optics, then sweeps, per chunk) and the two-kernel SW
    # (set-up, optics and layer R/T into the chunk scratch, then the adding sweeps, per chunk of day columns)
    lw_name = "lw3_optics_kernel+lw3_sweep_kernel"
    sw_name = "sw2_column_kernel" if mcfg.sw_sweep_chunk < 0 else "sw4_optics_kernel+sw4_sweep_kernel"
    dom = sw_name if sw_ms >= lw_ms else lw_name
    achieved = sw_tf if dom == sw_name else lw_tf
    traffic = None
    try:
        tr = json.loads(TRAFFIC.read_text())
        per = tr[dom]["dram_bytes_per_unit"]
        traffic = per * (nday if dom == sw_name else n)
    except (OSError, ValueError, KeyError):
        pass
    hbm_peak = float(pk.get("hbm_gbs", 6650.0))
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(cols, args.cpu_sample)
    parity = None
    if rank == 0 and ws == 1 and not args.no_parity:
        parity = parity_block(cols, mcfg, args.parity_sample)
    serving = None
    if ws == 1 and not args.no_serve and args.ncol is None:
        del mixed
        d.clear()
        out.clear()
        hin.clear()
        hout.clear()
        torch.cuda.empty_cache()
        serving = serving_block(10, args.serve_requests)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: 12 km NAM parent grid 954x835 columns x 61 radiation "
                                   f"layers (60 model layers), seed {seed}" + (" + rank offset" if ws > 1 else ""),
                       "columns": n, "day_columns": nday, "layers": cols.nlay,
                       "input_bytes": in_bytes, "output_bytes": out_bytes,
                       "l2": f"inputs ({in_bytes / 1e9:.1f} GB) larger than L2 (126 MB); no flush",
                       "parallelism": f"replicas x{ws} (one ensemble member per GPU)",
                       "lw_chunk": mcfg.lw_chunk, "sw_sweep_chunk": mcfg.sw_sweep_chunk},
            "roofline": {"bound": "fp32", "kernel": dom, "achieved": achieved, "peak": peak_tf,
                         "unit": "TFLOP/s", "frac": achieved / peak_tf, "traffic": traffic,
                         "peak_source": f"nominal FP32 pipe 148 SM x 128 lanes x 2 at the measured sm_max "
                                        f"{mhz:.0f} MHz (MEASURED_PEAKS.json holds no FP32 figure)",
                         "flops_per_unit": ops["sw_flops_per_daycol"] if dom == sw_name
                         else ops["lw_flops_per_col"],
                         "unit_of_work": "sunlit column" if dom == sw_name else "column",
                         "kernel_ms": {lw_name: lw_ms, "sw_prep": prof["prep_ms"] / max(prof["solves"], 1),
                                       sw_name: sw_ms},
                         "lw_tflops": lw_tf, "sw_tflops": sw_tf,
                         "hbm": {"achieved": (in_bytes + out_bytes) / (ms * 1e-3) / 1e9, "peak": hbm_peak,
                                 "unit": "GB/s", "frac": (in_bytes + out_bytes) / (ms * 1e-3) / 1e9 / hbm_peak}},
            "plain_fp64": fp64,
            "cpu_baseline": cpu,
            "parity": parity,
            "serving": serving,
            "e2e": {"value": ws * n / (ms_pipe * 1e-3), "unit": UNIT, "h2d_bytes_per_step": in_bytes,
                    "d2h_bytes_per_step": out_bytes, "ms_per_step": ms_pipe,
                    "how": "woof_nam_b200.pipeline.HostPipeline: every step copies its inputs from pinned host "
                           "memory and its outputs back, overlapped with the neighbouring steps' solves (two "
                           "device buffer sets)",
                    "serial": {"value": ws * n / (ms_e2e * 1e-3), "ms_per_step": ms_e2e,
                               "how": "RadSolver.solve between the two copies on one stream"}},
            "batch_c3": batch,
            "aerosols": aer,
            "front_end": front_leg,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
