"""The reference's radiation units bound to this library.

WOOF-NAM's radiation chain (namgpu/physics/rrtm/rrtm_call.py:246-365) runs, per chunk of rows, the grrad
front end, then phys-rrtm-grrad-sw, which calls the SW column unit ``phys_rrtm_sw_swrad.run(ctx,
has_htrswb)`` (phys_rrtm_grrad_sw.py:129,155), and phys-rrtm-grrad-lw, which scales the cloud paths by 1.5,
calls the LW column unit ``phys_rrtm_lw_lwrad.run(ctx)`` (phys_rrtm_grrad_lw.py:79) and restores them.
Both grrad units import the column unit by the module name held in ``SWRAD_MODULE`` / ``LWRAD_MODULE`` at
call time, so the units of this module drop in by name:

    phys_rrtm_grrad_sw.SWRAD_MODULE = "woof_nam_b200.swrad"
    phys_rrtm_grrad_lw.LWRAD_MODULE = "woof_nam_b200.lwrad"

or, for a whole radiation call, ``rrtm_call(ctx, args)`` below as the hook of
``phys_rad_driver.run(ctx, rrtm_call=...)`` (phys_rad_driver.py:171,255-262).

The units keep the reference's contract: inputs read from ``ctx.st`` by the reference's names, outputs
written to ``ctx.st`` under the reference's names through ``st.add``, all work on ``ctx.stream``, no host
synchronisation, a missing input refused by name with its producer.  Arrays may be CuPy or PyTorch CUDA
arrays (zero-copy through ``__cuda_array_interface__``), float32, C-contiguous, [field, level, JM, IM].
"""
from __future__ import annotations

import contextlib

from .solver import RadSolver, SolverConfig

# lwrad inputs: the unit's name, then the producer's state name (phys_rrtm_lw_lwrad.py:241-244), producer unit
LW_INPUTS = {
    "plyr": ("RAD_PLYR", "phys-rrtm-grrad-setup"), "plvl": ("RAD_PLVL", "phys-rrtm-grrad-setup"),
    "tlyr": ("RAD_TLYR", "phys-rrtm-grrad-setup"), "tlvl": ("TLVL", "phys-rrtm-grrad-gases"),
    "qlyr": ("QLYR", "phys-rrtm-grrad-gases"), "olyr": ("RAD_OLYR", "phys-rrtm-getozn"),
    "gasvmr": ("GASVMR", "phys-rrtm-getgases"), "clouds": ("RAD_CLOUDS", "phys-rrtm-grrad-clouds"),
    "tsfg": ("RAD_TSFG", "phys-rrtm-grrad-gases"), "sfcemis": ("sfcemis", "phys-rrtm-setemis"),
}
# swrad inputs (phys_rrtm_sw_swrad.py:104-116)
SW_INPUTS = {
    "plyr": ("RAD_PLYR", "phys-rrtm-grrad-setup"), "plvl": ("RAD_PLVL", "phys-rrtm-grrad-setup"),
    "tlyr": ("RAD_TLYR", "phys-rrtm-grrad-setup"), "qlyr": ("RAD_QLYR", "phys-rrtm-grrad-gases"),
    "olyr": ("RAD_OLYR", "phys-rrtm-getozn"), "gasvmr": ("GASVMR", "phys-rrtm-getgases"),
    "clouds": ("RAD_CLOUDS", "phys-rrtm-grrad-clouds"), "coszen": ("SW_COSZEN", "phys-rrtm-grrad-sw"),
    "sfcalb": ("SFCALB", "phys-rrtm-setalb"),
}
LW_FLUXES = ("topflw_upfxc", "topflw_upfx0", "sfcflw_upfxc", "sfcflw_upfx0", "sfcflw_dnfxc", "sfcflw_dnfx0")
SOLCON_DEFAULT = 1368.22
_KEY = "woof_nam_b200:solver"


def _torch():
    import torch
    return torch


def _fields(st) -> dict:
    return st.fields if hasattr(st, "fields") else st


def _get(st, unit: str, name: str, alias: str, producer: str):
    f = _fields(st)
    for k in (name, alias):
        if k in f:
            return f[k]
    raise KeyError(f"{unit}: input {name!r} ({alias}) is missing; its producer is {producer}")


def _as_tensor(x, name: str, unit: str):
    torch = _torch()
    t = x if isinstance(x, torch.Tensor) else torch.as_tensor(x, device="cuda")
    if not t.is_cuda or t.dtype != torch.float32:
        raise TypeError(f"{unit}: {name} must be a float32 CUDA array, got {t.dtype} on {t.device}")
    if not t.is_contiguous():
        raise ValueError(f"{unit}: {name} must be C-contiguous")
    return t


def _columns(st, unit: str, table: dict, jm: int, im: int, extra: dict) -> dict:
    cols = {}
    for k, (alias, producer) in table.items():
        t = _as_tensor(_get(st, unit, k, alias, producer), k, unit)
        if tuple(t.shape[-2:]) != (jm, im):
            raise ValueError(f"{unit}: {k} has trailing shape {tuple(t.shape[-2:])}, expected ({jm}, {im})")
        cols[k] = t.reshape(*t.shape[:-2], jm * im)
    for k, x in extra.items():
        if x is not None:
            t = _as_tensor(x, k, unit)
            cols[k] = t.reshape(*t.shape[:-2], jm * im)
    return cols


def _add(st, name: str, shape: tuple):
    """A float32 output array in the state: st.add(name, shape) when the state allocates (the reference's
    State), else a new zeroed CUDA tensor stored under name."""
    torch = _torch()
    if hasattr(st, "add"):
        return st.add(name, shape)
    t = torch.zeros(shape, dtype=torch.float32, device="cuda")
    st[name] = t
    return t


def _stream(ctx):
    torch = _torch()
    s = getattr(ctx, "stream", None)
    if s is None:
        return torch.cuda.current_stream()
    if isinstance(s, torch.cuda.Stream):
        return s
    return torch.cuda.ExternalStream(int(getattr(s, "ptr", 0)))


def _solver(ctx, parts: str, cpathfac: float, nlay: int) -> RadSolver:
    """One handle per (parts, cloud-path factor, layers), kept in ctx.tables (tables are shared per device)."""
    tabs = getattr(ctx, "tables", None)
    cache = tabs.setdefault(_KEY, {}) if tabs is not None else {}
    key = (parts, cpathfac, nlay)
    s = cache.get(key)
    if s is None:
        cfg = getattr(ctx, "cfg", None)
        s = RadSolver(SolverConfig(nlay=nlay, parts=parts, cpathfac=cpathfac,
                                   precision=getattr(cfg, "rad_precision", "mixed")))
        cache[key] = s
    return s


def _solcon(ctx) -> float:
    """solcon of this call: rrtm_call's record, else ctx.cfg.solcon, else NMMB's 1368.22
    (phys_rrtm_sw_swrad.py:297-304)."""
    tabs = getattr(ctx, "tables", None) or {}
    flags = tabs.get("rrtm_call_flags")
    if flags is not None and flags.get("solcon") is not None:
        return float(flags["solcon"])
    return float(getattr(getattr(ctx, "cfg", None), "solcon", SOLCON_DEFAULT))


def _faer(ctx, st, table_key: str, names: tuple):
    tabs = getattr(ctx, "tables", None) or {}
    if table_key in tabs:
        return tabs[table_key]
    f = _fields(st)
    for k in names:
        if k in f:
            return f[k]
    return None


def lwrad_run(ctx) -> dict:
    """Drop-in for phys_rrtm_lw_lwrad.run(ctx) (phys_rrtm_lw_lwrad.py:247-290): LW over every column of
    ctx.grid.  The clouds arrive already scaled by grrad-lw's cloud-path factor, so this unit applies none.
    Writes htlwc [LMK, JM, IM] and the six topflw_* / sfcflw_* [JM, IM] arrays; returns them as lwrad.run
    does (keys of LW_FLUXES and "hlwc")."""
    unit = "phys-rrtm-lw-lwrad"
    st = ctx.st
    g = ctx.grid
    jm, im, nlay = int(g.jm), int(g.im), int(g.lm) + 1
    cols = _columns(st, unit, LW_INPUTS, jm, im,
                    {"faerlw": _faer(ctx, st, "rrtm_faerlw", ("faerlw", "RAD_FAERLW"))})
    s = _solver(ctx, "lw", 1.0, nlay)
    stream = _stream(ctx)
    torch = _torch()
    cfg = getattr(ctx, "cfg", None)
    opt = {"hlw0": ("htlw0", (nlay, jm, im)) if getattr(cfg, "lhlw0", False) else None,
           "hlwb": ("htlwb", (16, nlay, jm, im)) if getattr(cfg, "lhlwb", False) else None,
           "lwflxprf": ("flwprf", (4, nlay + 1, jm, im)) if getattr(cfg, "lflxprf", False) else None}
    with torch.cuda.stream(stream):
        hl = _as_tensor(_add(st, "htlwc", (nlay, jm, im)), "htlwc", unit)
        out = s.alloc_outputs(jm * im)
        out["htlw"] = hl.reshape(nlay, jm * im)     # solved in place into the state's htlwc
        ret = {}
        for k, spec in opt.items():
            if spec is not None:
                name, shape = spec
                ret[k] = _as_tensor(_add(st, name, shape), name, unit)
                out[k] = ret[k].reshape(shape[0], -1) if len(shape) == 3 else ret[k].reshape(shape[0], shape[1], -1)
        s.solve(cols, _solcon(ctx), out, stream=stream)
        o = {}
        for i, n in enumerate(LW_FLUXES):
            dst = _as_tensor(_add(st, n, (jm, im)), n, unit)
            src = out["topflw"][i] if i < 2 else out["sfcflw"][i - 2]
            dst.view(-1).copy_(src)
            o[n] = dst
    o["hlwc"] = hl
    o["hlw0"], o["hlwb"], o["flxprf"] = ret.get("hlw0"), ret.get("hlwb"), ret.get("lwflxprf")
    return o


def swrad_run(ctx, has_htrswb: bool = False, nc: int = 0) -> dict:
    """Drop-in for phys_rrtm_sw_swrad.run(ctx, has_htrswb, nc) (phys_rrtm_sw_swrad.py:282-386): SW over
    the sunlit columns (SW_COSZEN >= 1e-4, the grrad-sw day predicate), zeros elsewhere.  Writes HTSWC
    [LMK, JM, IM], TOPFLX [3, JM, IM], SFCFLX [4, JM, IM] and, with ctx.cfg.lfdncmp, FDNCMP [6, JM, IM].
    The day list is built on the device inside the solve; nc (the reference's chunk size) has no effect
    on the result and is accepted for the signature.  With has_htrswb, ctx.cfg.lhsw0 and ctx.cfg.lflxprf
    it also writes HTSWB [14, LMK, JM, IM], HSW0 [LMK, JM, IM] and FLXPRF [4, LMK+1, JM, IM]."""
    unit = "phys-rrtm-sw-swrad"
    del nc
    cfg = getattr(ctx, "cfg", None)
    st = ctx.st
    g = ctx.grid
    jm, im, nlay = int(g.jm), int(g.im), int(g.lm) + 1
    cols = _columns(st, unit, SW_INPUTS, jm, im,
                    {"faersw": _faer(ctx, st, "rrtm_faersw", ("faersw", "RAD_FAERSW"))})
    s = _solver(ctx, "sw", 1.0, nlay)
    stream = _stream(ctx)
    torch = _torch()
    n = jm * im
    with torch.cuda.stream(stream):
        out = {}
        o = {"HTSWC": _as_tensor(_add(st, "HTSWC", (nlay, jm, im)), "HTSWC", unit),
             "TOPFLX": _as_tensor(_add(st, "TOPFLX", (3, jm, im)), "TOPFLX", unit),
             "SFCFLX": _as_tensor(_add(st, "SFCFLX", (4, jm, im)), "SFCFLX", unit)}
        out["htsw"] = o["HTSWC"].reshape(nlay, n)
        out["topfsw"] = o["TOPFLX"].reshape(3, n)
        out["sfcfsw"] = o["SFCFLX"].reshape(4, n)
        if getattr(cfg, "lfdncmp", False):
            o["FDNCMP"] = _as_tensor(_add(st, "FDNCMP", (6, jm, im)), "FDNCMP", unit)
            out["fdncmp"] = o["FDNCMP"].reshape(6, n)
        if has_htrswb:
            o["HTSWB"] = _as_tensor(_add(st, "HTSWB", (14, nlay, jm, im)), "HTSWB", unit)
            out["htswb"] = o["HTSWB"].reshape(14, nlay, n)
        if getattr(cfg, "lhsw0", False):
            o["HSW0"] = _as_tensor(_add(st, "HSW0", (nlay, jm, im)), "HSW0", unit)
            out["hsw0"] = o["HSW0"].reshape(nlay, n)
        if getattr(cfg, "lflxprf", False):
            o["FLXPRF"] = _as_tensor(_add(st, "FLXPRF", (4, nlay + 1, jm, im)), "FLXPRF", unit)
            out["swflxprf"] = o["FLXPRF"].reshape(4, nlay + 1, n)
        s.solve(cols, _solcon(ctx), out, stream=stream)
    return o


def column_solve(ctx, *, lslwr: bool = True, lsswr: bool = True) -> dict:
    """LW and SW of one radiation call in one launch set, for a chain that calls it in place of grrad-sw's
    swrad and grrad-lw's (scale clouds, lwrad, restore) block: the clouds are read unscaled and the LW
    kernel applies NAM's cloud-path factor 1.5 itself.  Writes the outputs of both units."""
    unit = "woof-nam-b200-column-solve"
    parts = "both" if (lslwr and lsswr) else "lw" if lslwr else "sw" if lsswr else None
    if parts is None:
        return {}
    st = ctx.st
    g = ctx.grid
    jm, im, nlay = int(g.jm), int(g.im), int(g.lm) + 1
    n = jm * im
    table = dict(LW_INPUTS) if lslwr else {}
    if lsswr:
        table.update(SW_INPUTS)
        if lslwr:
            table["qlyr"] = LW_INPUTS["qlyr"]
    extra = {"faerlw": _faer(ctx, st, "rrtm_faerlw", ("faerlw", "RAD_FAERLW")) if lslwr else None,
             "faersw": _faer(ctx, st, "rrtm_faersw", ("faersw", "RAD_FAERSW")) if lsswr else None}
    cols = _columns(st, unit, table, jm, im, extra)
    s = _solver(ctx, parts, 1.5, nlay)
    stream = _stream(ctx)
    torch = _torch()
    o = {}
    with torch.cuda.stream(stream):
        out = {k: v for k, v in s.alloc_outputs(n).items() if k in ("topflw", "sfcflw")}
        if lslwr:
            o["htlwc"] = _as_tensor(_add(st, "htlwc", (nlay, jm, im)), "htlwc", unit)
            out["htlw"] = o["htlwc"].reshape(nlay, n)
        if lsswr:
            for k, (name, rows) in {"htsw": ("HTSWC", nlay), "topfsw": ("TOPFLX", 3), "sfcfsw": ("SFCFLX", 4)}.items():
                o[name] = _as_tensor(_add(st, name, (rows, jm, im)), name, unit)
                out[k] = o[name].reshape(rows, n)
        s.solve(cols, _solcon(ctx), out, stream=stream)
        if lslwr:
            for i, name in enumerate(LW_FLUXES):
                o[name] = _as_tensor(_add(st, name, (jm, im)), name, unit)
                o[name].view(-1).copy_(out["topflw"][i] if i < 2 else out["sfcflw"][i - 2])
    return o


POST_OUTPUTS_2D = ("RLWIN", "RSWIN", "RSWINC", "RSWOUT", "RLWTOA", "RSWTOA", "CZMEAN", "SIGT4", "CFRACL",
                   "CFRACM", "CFRACH", "ACFRST", "ACFRCV", "NCFRST", "NCFRCV")


def driver_post_run(ctx, *, icwp: int = 1, ntimestep: int | None = None, lssav: bool = True,
                    cncld: bool = True) -> None:
    """Drop-in for phys_rrtm_driver_post.run (phys_rrtm_driver_post.py:121-202) on NAM's ICWP /= -1 path:
    one rad_post_outputs launch reads the grrad outputs by the reference's names (htrlw, HTRSW, cldcov,
    cldsa, GRRAD_COSZDG_V, GRRAD_COSZEN_V, sfcflw_dnfxc, topflw_upfxc, SFCFSW, TOPFSW,
    ctx.tables["rrtm_driver_call"]["CU_CLOUD"]) and the state (CW, T), and writes RLWTT, RSWTT, CLDFRA,
    CSMID, the surface / TOA fields, the cloud fractions and accumulators, COSZDG and, on LW steps
    (NTIMESTEP mod NRADL == 0), SIGT4.  lssav false and the ICWP == -1 (old NAM/GFDL) cloud block are
    refused."""
    unit = "phys-rrtm-driver-post"
    del cncld                 # read only by the ICWP == -1 block
    if not lssav:
        raise NotImplementedError(f"{unit}: lssav=False makes the Fortran STOP; not run")
    if icwp == -1:
        raise NotImplementedError(f"{unit}: the ICWP == -1 (old NAM/GFDL) cloud block is not built")
    torch = _torch()
    st, g = ctx.st, ctx.grid
    jm, im, lm = int(g.jm), int(g.im), int(g.lm)
    n = jm * im
    nts = int(ctx.ntimestep if ntimestep is None else ntimestep)
    lw_step = nts % int(getattr(ctx.cfg, "nradl", 48)) == 0
    f = _fields(st)

    def need(name, owner):
        if name not in f:
            raise KeyError(f"{unit}: ctx.st['{name}'] is missing (written by {owner}, which has not run)")
        return _as_tensor(f[name], name, unit) if name not in ("NCFRST", "NCFRCV") else f[name]

    lw_post = "phys-rrtm-grrad-lw (post_heat / post_flux)"
    sfcfsw = need("SFCFSW", "phys-rrtm-grrad-sw").reshape(4, n)
    topfsw = need("TOPFSW", "phys-rrtm-grrad-sw").reshape(3, n)
    cu = (getattr(ctx, "tables", None) or {}).get("rrtm_driver_call", {}).get("CU_CLOUD")
    if cu is None:
        raise KeyError(f"{unit}: ctx.tables['rrtm_driver_call']['CU_CLOUD'] is missing (written by "
                       "phys-rrtm-driver-call, which has not run)")
    cu = torch.as_tensor(cu, device="cuda")
    if cu.dtype != torch.int32:
        raise TypeError(f"{unit}: CU_CLOUD must be int32, got {cu.dtype}")
    inp = {"hlw": need("htrlw", lw_post).reshape(lm, n), "swh": need("HTRSW", "phys-rrtm-grrad-sw").reshape(lm, n),
           "coszdg_v": need("GRRAD_COSZDG_V", "phys-rrtm-coszmn").reshape(n),
           "coszen_v": need("GRRAD_COSZEN_V", "phys-rrtm-coszmn").reshape(n),
           "sfcflw_dnfxc": need("sfcflw_dnfxc", "phys-rrtm-lw-lwrad").reshape(n),
           "topflw_upfxc": need("topflw_upfxc", "phys-rrtm-lw-lwrad").reshape(n),
           "sfcfsw_upfxc": sfcfsw[0], "sfcfsw_dnfxc": sfcfsw[1], "sfcfsw_dnfx0": sfcfsw[3], "topfsw_upfxc": topfsw[0],
           "cldcov": need("cldcov", lw_post).reshape(lm, n), "cldsa": need("cldsa", lw_post).reshape(5, n),
           "cw": need("CW", "the state").reshape(lm, n), "t": need("T", "the state").reshape(lm, n),
           "cu_cloud": cu.reshape(n)}
    out = {"rlwtt": need("RLWTT", "the state").reshape(lm, n), "rswtt": need("RSWTT", "the state").reshape(lm, n),
           "cldfra": need("CLDFRA", "the state").reshape(lm, n),
           "csmid": _as_tensor(_add(st, "CSMID", (lm, jm, im)), "CSMID", unit).reshape(lm, n),
           "coszdg": _as_tensor(_add(st, "COSZDG", (jm, im)), "COSZDG", unit).reshape(n)}
    for k in POST_OUTPUTS_2D:
        t = need(k, "the state")
        if k in ("NCFRST", "NCFRCV"):
            t = torch.as_tensor(t, device="cuda")
            if t.dtype != torch.int32:
                raise TypeError(f"{unit}: {k} must be int32, got {t.dtype}")
        out[k.lower()] = t.reshape(n)
    s = _solver(ctx, "both", 1.5, lm + 1)
    s.post_outputs(inp, out, lm, kd=0, cloud_block=True, lw_step=lw_step, stream=_stream(ctx))


_MONTH = (31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31)


def rdtemp_run(ctx) -> None:
    """Drop-in for drv_rdtemp.run (namgpu/steps/drv_rdtemp.py): the radiative temperature change of every
    step, one rad_rdtemp launch.  Reads GLAT, GLON, CZMEAN [JM, IM], RSWTT, RLWTT [LM, JM, IM], updates T
    in place and writes CZEN on the tile.  Calendar (JULDAY, JULYR, start hour, leap flag) from ctx.start,
    derived once and kept in ctx.tables["RDTEMP_CAL"]; the tile and interior from
    ctx.tables["drv_loop_limits"] (ITS, ITE, JTS, JTE, ITS_B1, ITE_B1, JTS_B1, JTE_B1, 1-based) when
    present, else the whole grid and its interior without the edge rows and columns."""
    unit = "drv-rdtemp"
    st, g = ctx.st, ctx.grid
    im, jm, lm = int(g.im), int(g.jm), int(g.lm)
    tabs = ctx.tables
    cal = tabs.get("RDTEMP_CAL")
    if cal is None:
        s0 = getattr(ctx, "start", None)
        if s0 is None:
            raise RuntimeError(f"{unit}: ctx.start (the initial time) is not set")
        month = list(_MONTH)
        leap = s0.year % 4 == 0
        if leap:
            month[1] = 29
        cal = (sum(month[: s0.month - 1]) + s0.day, int(s0.year), int(s0.hour), int(leap))
        tabs["RDTEMP_CAL"] = cal
    lim = tabs.get("drv_loop_limits") or {"ITS": 1, "ITE": im, "JTS": 1, "JTE": jm, "ITS_B1": 2, "ITE_B1": im - 1,
                                           "JTS_B1": 2, "JTE_B1": jm - 1}
    f = _fields(st)

    def need(name, shape):
        if name not in f:
            raise KeyError(f"{unit}: ctx.st['{name}'] is missing")
        t = _as_tensor(f[name], name, unit)
        if tuple(t.shape) != shape:
            raise ValueError(f"{unit}: {name} has shape {tuple(t.shape)}, expected {shape}")
        return t

    czen = _as_tensor(_add(st, "CZEN", (jm, im)) if "CZEN" not in f else f["CZEN"], "CZEN", unit)
    p = {"ntsd": int(ctx.ntimestep), "dt": float(ctx.dt), "julday": int(cal[0]), "julyr": int(cal[1]),
         "ihrst": int(cal[2]), "leap_seen": int(cal[3]), "glat": need("GLAT", (jm, im)), "glon": need("GLON", (jm, im)),
         "czmean": need("CZMEAN", (jm, im)), "rswtt": need("RSWTT", (lm, jm, im)), "rlwtt": need("RLWTT", (lm, jm, im)),
         "czen": czen, "t": need("T", (lm, jm, im)), "im": im, "jm": jm, "lm": lm,
         "its": lim["ITS"], "ite": lim["ITE"], "jts": lim["JTS"], "jte": lim["JTE"],
         "its_b1": lim["ITS_B1"], "ite_b1": lim["ITE_B1"], "jts_b1": lim["JTS_B1"], "jte_b1": lim["JTE_B1"]}
    _solver(ctx, "both", 1.5, lm + 1).rdtemp(p, stream=_stream(ctx))


# grrad's setaer inputs: the unit's name, the grrad-setup / model state name (phys_rrtm_grrad_aerosols.py:12-22)
AER_INPUTS = {
    "plvl": ("RAD_PLVL", "phys-rrtm-grrad-setup"), "plyr": ("RAD_PLYR", "phys-rrtm-grrad-setup"),
    "tlyr": ("RAD_TLYR", "phys-rrtm-grrad-setup"), "qlyr": ("RAD_QLYR", "phys-rrtm-grrad-setup"),
    "rhly": ("RAD_RHLY", "phys-rrtm-grrad-setup"), "xlon": ("XLON", "the model grid"),
    "xlat": ("XLAT", "the model grid"), "slmsk": ("SLMSK", "the model state"),
}


def _aer_month(ctx) -> int:
    """The month of the aerosol climatology: ctx.tables["aer_month"] when the driver's calendar sets it
    (aer_update runs at month changes), else ctx.clock.idate[1], else the month of ctx.start."""
    tabs = getattr(ctx, "tables", None) or {}
    if tabs.get("aer_month"):
        return int(tabs["aer_month"])
    clock = getattr(ctx, "clock", None)
    if clock is not None and getattr(clock, "idate", None) is not None:
        return int(clock.idate[1])
    start = getattr(ctx, "start", None)
    if start is None:
        raise RuntimeError("phys-rrtm-grrad-aerosols: no month (ctx.tables['aer_month'], ctx.clock or ctx.start)")
    return int(start.month)


# Slots of rad_initialize's flag vector (namgpu/kernels/phys_rrtm_rad_initialize.cu:99-108).
RI_IAERFLG, RI_LASWFLG, RI_LALWFLG, RI_LAVOFLG, RI_IVFLIP = 4, 5, 6, 7, 25


def _aer_flags(ctx) -> dict:
    """setaer's module state (phys_rrtm_grrad_aerosols.py:63-85): ctx.tables["aer_state"] when grrad's aerosol
    unit built it, else rad_initialize's flags in ctx.tables["rad_physparam"], else NAM's iaer = 11 (SW and LW
    aerosol, no volcanic term).  kyrsav / kmonsav come from ctx.tables["aer_volc"] (default 1, 1)."""
    tabs = getattr(ctx, "tables", None) or {}
    st = tabs.get("aer_state")
    if st is None:
        p = tabs.get("rad_physparam")
        if p is not None:
            import numpy as np
            p = np.asarray(p.get() if hasattr(p, "get") and not isinstance(p, dict) else p)
            st = {"iaerflg": int(p[RI_IAERFLG]), "laswflg": bool(p[RI_LASWFLG]), "lalwflg": bool(p[RI_LALWFLG]),
                  "lavoflg": bool(p[RI_LAVOFLG]), "ivflip": int(p[RI_IVFLIP]) if p.size > RI_IVFLIP else 0}
        else:
            st = {"iaerflg": 11, "laswflg": True, "lalwflg": True, "lavoflg": False, "ivflip": 0}
        volc = tabs.get("aer_volc")
        st = dict(st, kyrsav=int(getattr(volc, "kyrsav", 1)), kmonsav=int(getattr(volc, "kmonsav", 1)))
    return st


def grrad_aerosols_run(ctx, *, lsswr: bool = True, lslwr: bool = True) -> dict:
    """Drop-in for phys_rrtm_grrad_aerosols.run(ctx, lsswr=, lslwr=) (phys_rrtm_grrad_aerosols.py:124-136):
    setaer's aerosol optics of every column of ctx.grid, written to ctx.tables["rrtm_faersw"]
    [3, 14, LMK, JM, IM] and ["rrtm_faerlw"] [3, 16, LMK, JM, IM], where lwrad / swrad read them, under the
    module flags of _aer_flags (phys_rrtm_setaer.py:150-192): zeros unless a radiation call is due and iaerflg
    > 0; the climatological optics of the calls the flags allow (the month's tables (re)loaded when the month
    changes); then, with lavoflg, the volcanic term from ctx.tables["aer_ivolae"] (int32 [10, 4, 12])."""
    from .aerosols import Aerosols, volcanic
    unit = "phys-rrtm-grrad-aerosols"
    st, g = ctx.st, ctx.grid
    jm, im, nlay = int(g.jm), int(g.im), int(g.lm) + 1
    cols = {}
    for k, (alias, producer) in AER_INPUTS.items():
        t = _as_tensor(_get(st, unit, k, alias, producer), k, unit)
        if tuple(t.shape[-2:]) != (jm, im):
            raise ValueError(f"{unit}: {k} has trailing shape {tuple(t.shape[-2:])}, expected ({jm}, {im})")
        cols[k] = t.reshape(*t.shape[:-2], jm * im)
    s = _solver(ctx, "both", 1.5, nlay)
    tabs = ctx.tables
    aer = tabs.get(_KEY + ":aerosols")
    month = _aer_month(ctx)
    if aer is None or aer.solver is not s:
        aer = Aerosols(s, month)
        tabs[_KEY + ":aerosols"] = aer
    elif aer.month != month:
        aer.load(month)
    torch = _torch()
    fsw, flw = tabs.get("rrtm_faersw"), tabs.get("rrtm_faerlw")
    if fsw is None or tuple(fsw.shape) != (3, 14, nlay, jm, im):
        fsw = torch.zeros((3, 14, nlay, jm, im), dtype=torch.float32, device="cuda")
        flw = torch.zeros((3, 16, nlay, jm, im), dtype=torch.float32, device="cuda")
    stream = _stream(ctx)
    out = (fsw.view(3, 14, nlay, jm * im), flw.view(3, 16, nlay, jm * im))
    fl = _aer_flags(ctx)
    laersw, laerlw = bool(lsswr and fl["laswflg"]), bool(lslwr and fl["lalwflg"])
    with torch.cuda.stream(stream):
        if fl["iaerflg"] > 0 and (lsswr or lslwr) and (fl["laswflg"] or fl["lalwflg"]):
            aer.optics(cols, cols["rhly"], cols["xlon"], cols["xlat"], cols["slmsk"], out=out, stream=stream,
                       ivflip=int(fl.get("ivflip", 0)))
            if not laersw:
                fsw.zero_()
            if not laerlw:
                flw.zero_()
        else:
            fsw.zero_()
            flw.zero_()
    if fl["iaerflg"] > 0 and (lsswr or lslwr) and fl["lavoflg"]:
        add_sw = bool(lsswr) if fl["iaerflg"] == 100 else laersw
        add_lw = bool(lslwr) if fl["iaerflg"] == 100 else laerlw
        iv = tabs.get("aer_ivolae")
        if iv is None:
            raise RuntimeError(f"{unit}: lavoflg needs ctx.tables['aer_ivolae'] (int32 [10, 4, 12])")
        if hasattr(iv, "get") and not isinstance(iv, dict):
            iv = iv.get()
        volcanic(s, cols["plvl"], cols["xlat"], iv, fl["kyrsav"], fl["kmonsav"], out, ivflip=int(fl.get("ivflip", 0)),
                 add_sw=add_sw, add_lw=add_lw, stream=stream)
    tabs["rrtm_faersw"], tabs["rrtm_faerlw"] = fsw, flw
    return {"faersw": fsw, "faerlw": flw}


@contextlib.contextmanager
def bound_units():
    """Bind the reference's grrad units to this library's column units for the duration of the block."""
    from namgpu.physics.rrtm import phys_rrtm_grrad_lw as glw
    from namgpu.physics.rrtm import phys_rrtm_grrad_sw as gsw
    old = (glw.LWRAD_MODULE, gsw.SWRAD_MODULE)
    glw.LWRAD_MODULE, gsw.SWRAD_MODULE = "woof_nam_b200.lwrad", "woof_nam_b200.swrad"
    try:
        yield
    finally:
        glw.LWRAD_MODULE, gsw.SWRAD_MODULE = old


def rrtm_call(ctx, args: dict) -> None:
    """The rrtm_call hook of phys_rad_driver.run (phys_rad_driver.py:255-262): the reference's radiation
    chain (namgpu.physics.rrtm.rrtm_call.run) with its LW and SW column units bound to this library."""
    from namgpu.physics.rrtm import rrtm_call as chain
    with bound_units():
        chain.run(ctx, args)
