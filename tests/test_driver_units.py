"""The reference-facing units (woof_nam_b200.lwrad / swrad / driver.column_solve) on a state laid out as
the reference's: inputs by the reference's names in [field, level, JM, IM], outputs written back by name.
They equal the solver called directly."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from woof_nam_b200 import driver
from woof_nam_b200.columns import make_columns

JM, IM = 7, 50


class State:
    """The reference's State surface the units use: fields by name, st[name], st.add(name, shape)."""

    def __init__(self):
        self.fields = {}

    def __getitem__(self, k):
        return self.fields[k]

    def __setitem__(self, k, v):
        self.fields[k] = v

    def add(self, name, shape):
        import torch
        t = self.fields.get(name)
        if t is None or tuple(t.shape) != tuple(shape):
            t = torch.zeros(shape, dtype=torch.float32, device="cuda")
            self.fields[name] = t
        return t


def _ctx(cols, device="cuda", cloud_scale=None):
    import torch
    st = State()
    names = {"plyr": ("RAD_PLYR",), "plvl": ("RAD_PLVL",), "tlyr": ("RAD_TLYR",), "tlvl": ("TLVL",),
             "qlyr": ("QLYR", "RAD_QLYR"), "olyr": ("RAD_OLYR",), "gasvmr": ("GASVMR",),
             "clouds": ("RAD_CLOUDS",), "tsfg": ("RAD_TSFG",), "sfcemis": ("sfcemis",),
             "coszen": ("SW_COSZEN",), "sfcalb": ("SFCALB",)}
    for k, aliases in names.items():
        a = np.ascontiguousarray(getattr(cols, k), dtype=np.float32)
        t = torch.from_numpy(a.reshape(*a.shape[:-1], JM, IM).copy()).to(device)
        if k == "clouds" and cloud_scale is not None:
            t[1] *= cloud_scale       # cloud liquid path (Fortran index 2)
            t[3] *= cloud_scale       # cloud ice path (Fortran index 4)
        for n in aliases:
            st[n] = t
    grid = SimpleNamespace(jm=JM, im=IM, lm=cols.nlay - 1)
    cfg = SimpleNamespace(solcon=cols.solcon, lfdncmp=True)
    return SimpleNamespace(st=st, grid=grid, tables={}, cfg=cfg, stream=None)


def test_missing_input_named_with_producer():
    ctx = SimpleNamespace(st=State(), grid=SimpleNamespace(jm=JM, im=IM, lm=60), tables={}, cfg=None, stream=None)
    with pytest.raises(KeyError, match="RAD_PLYR.*phys-rrtm-grrad-setup"):
        driver.lwrad_run(ctx)
    with pytest.raises(KeyError, match="RAD_PLYR.*phys-rrtm-grrad-setup"):
        driver.swrad_run(ctx)


@pytest.mark.gpu
def test_units_write_optional_outputs():
    """swrad with has_htrswb, lhsw0, lflxprf and lwrad with lhlw0, lhlwb, lflxprf write HTSWB / HSW0 / FLXPRF
    and htlwb / htlw0 / flwprf by the reference's names, equal to the solver's optional outputs."""
    import torch
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(JM * IM, 79)
    flags = dict(lhsw0=True, lhswb=True, lhlw0=True, lhlwb=True, lflxprf=True)
    ctx = _ctx(cols)
    ctx.cfg.lhsw0 = ctx.cfg.lflxprf = ctx.cfg.lhlw0 = ctx.cfg.lhlwb = True
    o = driver.swrad_run(ctx, has_htrswb=True)
    torch.cuda.synchronize()
    r = RadSolver(precision="mixed", parts="sw", **flags).solve_host(cols)
    for name, key in (("HTSWB", "htswb"), ("HSW0", "hsw0"), ("FLXPRF", "swflxprf")):
        got = o[name].cpu().numpy()
        assert np.array_equal(got.reshape(r[key].shape), r[key]), name
        assert ctx.st.fields[name] is o[name]
    ctx = _ctx(cols, cloud_scale=np.float32(1.5))
    ctx.cfg.lhlw0 = ctx.cfg.lhlwb = ctx.cfg.lflxprf = True
    o = driver.lwrad_run(ctx)
    torch.cuda.synchronize()
    r = RadSolver(precision="mixed", parts="lw", cpathfac=1.0, **flags).solve_host(_scaled(cols))
    for name, key, out in (("htlw0", "hlw0", "hlw0"), ("htlwb", "hlwb", "hlwb"), ("flwprf", "lwflxprf", "flxprf")):
        assert np.array_equal(o[out].cpu().numpy().reshape(r[key].shape), r[key]), name
        assert ctx.st.fields[name] is o[out]


def _scaled(cols):
    """The request with grrad-lw's cloud-path factor applied to the liquid and ice paths."""
    from woof_nam_b200.columns import Columns
    kw = {f: np.array(getattr(cols, f)) for f in Columns.FIELDS}
    kw["clouds"][1] *= np.float32(1.5)
    kw["clouds"][3] *= np.float32(1.5)
    return Columns(**kw, solcon=cols.solcon, diagnostic_clouds=cols.diagnostic_clouds)


@pytest.mark.gpu
def test_units_equal_solver():
    import torch
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(JM * IM, 77)
    s = RadSolver(precision="mixed")
    ref = s.solve(s.to_device(cols), cols.solcon)
    torch.cuda.synchronize()
    r = {k: v.cpu().numpy() for k, v in ref.items()}

    # one launch set for both parts
    ctx = _ctx(cols)
    o = driver.column_solve(ctx)
    torch.cuda.synchronize()
    st = ctx.st
    assert np.array_equal(st["htlwc"].cpu().numpy().reshape(cols.nlay, -1), r["htlw"])
    assert np.array_equal(st["HTSWC"].cpu().numpy().reshape(cols.nlay, -1), r["htsw"])
    assert np.array_equal(st["TOPFLX"].cpu().numpy().reshape(3, -1), r["topfsw"])
    assert np.array_equal(st["SFCFLX"].cpu().numpy().reshape(4, -1), r["sfcfsw"])
    for i, n in enumerate(driver.LW_FLUXES):
        want = r["topflw"][i] if i < 2 else r["sfcflw"][i - 2]
        assert np.array_equal(o[n].cpu().numpy().reshape(-1), want), n

    # the SW unit alone
    ctx = _ctx(cols)
    o = driver.swrad_run(ctx)
    torch.cuda.synchronize()
    assert np.array_equal(o["HTSWC"].cpu().numpy().reshape(cols.nlay, -1), r["htsw"])
    assert np.array_equal(o["FDNCMP"].cpu().numpy().reshape(6, -1), r["fdncmp"])
    assert "htlwc" not in ctx.st.fields

    # the LW unit alone, on clouds grrad-lw has already scaled by 1.5: equal up to the rounding of where
    # the scaling happens, far inside 0.01 K/day and 0.05 W/m^2
    ctx = _ctx(cols, cloud_scale=np.float32(1.5))
    o = driver.lwrad_run(ctx)
    torch.cuda.synchronize()
    ht = o["hlwc"].cpu().numpy().reshape(cols.nlay, -1).astype(np.float64)
    assert np.max(np.abs(ht - r["htlw"])) * 86400.0 < 1e-3
    for i, n in enumerate(driver.LW_FLUXES):
        want = r["topflw"][i] if i < 2 else r["sfcflw"][i - 2]
        assert np.max(np.abs(o[n].cpu().numpy().reshape(-1) - want)) < 5e-3, n
    assert "HTSWC" not in ctx.st.fields


@pytest.mark.gpu
def test_lw_only_and_sw_only_steps():
    """column_solve on a step where only lslwr (or only lsswr) holds runs that part alone."""
    import torch
    cols = make_columns(JM * IM, 78)
    ctx = _ctx(cols)
    driver.column_solve(ctx, lslwr=True, lsswr=False)
    torch.cuda.synchronize()
    assert "htlwc" in ctx.st.fields and "HTSWC" not in ctx.st.fields
    ctx2 = _ctx(cols)
    driver.column_solve(ctx2, lslwr=False, lsswr=True)
    torch.cuda.synchronize()
    assert "HTSWC" in ctx2.st.fields and "htlwc" not in ctx2.st.fields
    ctx3 = _ctx(cols)
    driver.column_solve(ctx3)
    torch.cuda.synchronize()
    assert torch.equal(ctx.st["htlwc"], ctx3.st["htlwc"])
    assert torch.equal(ctx2.st["HTSWC"], ctx3.st["HTSWC"])


@pytest.mark.gpu
def test_driver_post_equals_oracle():
    """driver_post_run on a state under the reference's names gives the oracle's post step."""
    import torch
    from oracle import post
    lm, jm, im = 60, 4, 33
    n = jm * im
    inp, state = post.make_case(n, lm, 9)
    ref = post.post_outputs(inp, state, lm, lw_step=True)
    st = State()
    t = lambda a, *shape: torch.from_numpy(np.ascontiguousarray(a).reshape(*shape)).cuda()  # noqa: E731
    st["htrlw"], st["HTRSW"] = t(inp["hlw"], lm, jm, im), t(inp["swh"], lm, jm, im)
    st["cldcov"], st["cldsa"] = t(inp["cldcov"], lm, jm, im), t(inp["cldsa"], 5, jm, im)
    st["GRRAD_COSZDG_V"], st["GRRAD_COSZEN_V"] = t(inp["coszdg_v"], jm, im), t(inp["coszen_v"], jm, im)
    st["sfcflw_dnfxc"], st["topflw_upfxc"] = t(inp["sfcflw_dnfxc"], jm, im), t(inp["topflw_upfxc"], jm, im)
    sfc = np.stack([inp["sfcfsw_upfxc"], inp["sfcfsw_dnfxc"], np.zeros(n, np.float32), inp["sfcfsw_dnfx0"]])
    top = np.stack([inp["topfsw_upfxc"], np.zeros(n, np.float32), np.zeros(n, np.float32)])
    st["SFCFSW"], st["TOPFSW"] = t(sfc, 4, jm, im), t(top, 3, jm, im)
    st["CW"], st["T"] = t(inp["cw"], lm, jm, im), t(inp["t"], lm, jm, im)
    for k in ("RLWTT", "RSWTT", "CLDFRA"):
        st[k] = torch.zeros((lm, jm, im), dtype=torch.float32, device="cuda")
    for k in driver.POST_OUTPUTS_2D:
        low = k.lower()
        st[k] = t(state[low], jm, im) if low in state else torch.zeros((jm, im), dtype=torch.float32, device="cuda")
    ctx = SimpleNamespace(st=st, grid=SimpleNamespace(jm=jm, im=im, lm=lm), cfg=SimpleNamespace(nradl=48),
                          tables={"rrtm_driver_call": {"CU_CLOUD": t(inp["cu_cloud"], jm, im)}}, stream=None,
                          ntimestep=96)
    driver.driver_post_run(ctx)
    torch.cuda.synchronize()
    for k in ("rlwtt", "rswtt", "cldfra", "csmid", "coszdg"):
        assert np.array_equal(st[k.upper()].cpu().numpy().reshape(ref[k].shape), ref[k]), k
    for k in driver.POST_OUTPUTS_2D:
        assert np.array_equal(st[k].cpu().numpy().reshape(-1), ref[k.lower()]), k
    assert np.array_equal(st["cldcov"].cpu().numpy().reshape(lm, n), ref["cldcov"])


@pytest.mark.gpu
def test_rdtemp_unit_equals_oracle():
    """rdtemp_run on a state under the reference's names (GLAT, GLON, CZMEAN, RSWTT, RLWTT, T, CZEN)."""
    import datetime
    import torch
    from oracle import rdtemp
    im, jm, lm = 40, 30, 12
    p = rdtemp.make_case(im, jm, lm, 4, ntsd=240, julday=59, julyr=2026, ihrst=6)
    ref = rdtemp.rdtemp(p)
    st = State()
    for name, key in (("GLAT", "glat"), ("GLON", "glon"), ("CZMEAN", "czmean"), ("RSWTT", "rswtt"),
                      ("RLWTT", "rlwtt"), ("T", "t"), ("CZEN", "czen")):
        st[name] = torch.from_numpy(np.ascontiguousarray(p[key])).cuda()
    ctx = SimpleNamespace(st=st, grid=SimpleNamespace(jm=jm, im=im, lm=lm), cfg=None, tables={}, stream=None,
                          ntimestep=240, dt=p["dt"], start=datetime.datetime(2026, 2, 28, 6))
    driver.rdtemp_run(ctx)
    torch.cuda.synchronize()
    assert ctx.tables["RDTEMP_CAL"] == (59, 2026, 6, 0)
    assert np.max(np.abs(st["CZEN"].cpu().numpy() - ref["czen"])) < 3e-5      # float angle resolution
    changed = st["T"].cpu().numpy() != p["t"]
    assert changed[:, 1:-1, 1:-1].any() and not changed[:, 0, :].any()       # interior only


@pytest.mark.gpu
def test_grrad_aerosols_unit_feeds_the_solve():
    """grrad_aerosols.run on a state under the reference's names (RAD_PLVL, RAD_PLYR, RAD_TLYR, RAD_QLYR,
    RAD_RHLY, XLON, XLAT, SLMSK) writes rrtm_faersw / rrtm_faerlw equal to the aerosol optics called
    directly, and the column solve then reads them as the solver does the same optics."""
    import datetime

    import torch
    from woof_nam_b200 import aerosols, grrad_aerosols
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(JM * IM, 23)
    ai = aerosols.make_inputs(cols, 6, "nam")
    ctx = _ctx(cols)
    ctx.start = datetime.datetime(2026, 5, 1)
    for name, key in (("RAD_RHLY", "rhly"),):
        ctx.st[name] = torch.from_numpy(ai[key].reshape(cols.nlay, JM, IM).copy()).cuda()
    for name, key in (("XLON", "xlon"), ("XLAT", "xlat"), ("SLMSK", "slmsk")):
        ctx.st[name] = torch.from_numpy(ai[key].reshape(JM, IM).copy()).cuda()
    o = grrad_aerosols.run(ctx, lsswr=True, lslwr=True)
    driver.column_solve(ctx)
    torch.cuda.synchronize()
    s = RadSolver()
    dev = s.to_device(cols)
    aer = aerosols.Aerosols(s, 5)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in ai.items()}
    fsw, flw = aer.optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"])
    torch.cuda.synchronize()
    assert torch.equal(o["faersw"].reshape(fsw.shape), fsw) and torch.equal(o["faerlw"].reshape(flw.shape), flw)
    dev["faersw"], dev["faerlw"] = fsw, flw
    ref = s.solve(dev, cols.solcon)
    torch.cuda.synchronize()
    assert torch.equal(ctx.st["htlwc"].reshape(ref["htlw"].shape), ref["htlw"])
    assert torch.equal(ctx.st["HTSWC"].reshape(ref["htsw"].shape), ref["htsw"])


@pytest.mark.gpu
def test_grrad_aerosols_unit_flags_and_volcanic():
    """The unit under rad_initialize's flags (ctx.tables["rad_physparam"]): iaer = 111 adds the volcanic term
    from ctx.tables["aer_ivolae"] for the year and month of ctx.tables["aer_volc"] to the climatological
    optics of the calls that are due (here SW only, so the LW optics are zeros), as setaer does
    (phys_rrtm_setaer.py:150-192); iaer = 0 gives zeros."""
    import datetime
    from types import SimpleNamespace

    import torch
    from woof_nam_b200 import aerosols, grrad_aerosols
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(JM * IM, 29)
    ai = aerosols.make_inputs(cols, 7, "globe")
    ctx = _ctx(cols)
    ctx.start = datetime.datetime(2026, 9, 1)
    ctx.st["RAD_RHLY"] = torch.from_numpy(ai["rhly"].reshape(cols.nlay, JM, IM).copy()).cuda()
    for name, key in (("XLON", "xlon"), ("XLAT", "xlat"), ("SLMSK", "slmsk")):
        ctx.st[name] = torch.from_numpy(ai[key].reshape(JM, IM).copy()).cuda()
    iv = np.random.default_rng(2).integers(0, 600, (10, 4, 12)).astype(np.int32)
    flags = np.zeros(26, np.int32)
    flags[4:8] = (111, 1, 1, 1)                   # iaerflg, laswflg, lalwflg, lavoflg
    ctx.tables.update(rad_physparam=flags, aer_ivolae=iv, aer_volc=SimpleNamespace(kyrsav=1994, kmonsav=9))
    o = grrad_aerosols.run(ctx, lsswr=True, lslwr=False)
    torch.cuda.synchronize()
    s = RadSolver()
    dev = s.to_device(cols)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in ai.items()}
    fsw, flw = aerosols.Aerosols(s, 9).optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"])
    aerosols.volcanic(s, dev["plvl"], t["xlat"], iv, 1994, 9, (fsw, flw), add_lw=False)
    torch.cuda.synchronize()
    assert torch.equal(o["faersw"].reshape(fsw.shape), fsw)
    assert not o["faerlw"].any()
    flags[4:8] = (0, 0, 0, 0)
    ctx.tables.pop("aer_state", None)
    o = grrad_aerosols.run(ctx, lsswr=True, lslwr=True)
    torch.cuda.synchronize()
    assert not o["faersw"].any() and not o["faerlw"].any()


def test_aerosol_module_flags():
    """setaer's module state as the aerosol unit reads it (no GPU): rad_initialize's flag vector, iaer = 11 (NAM),
    111 (with the volcanic term), 100 (volcanic only) and 0; grrad's aer_state when present; the defaults."""
    def ctx(**tables):
        return SimpleNamespace(tables=tables)

    assert driver._aer_flags(ctx()) == {"iaerflg": 11, "laswflg": True, "lalwflg": True, "lavoflg": False,
                                        "ivflip": 0, "kyrsav": 1, "kmonsav": 1}
    for iaer, sw, lw, vo in ((11, 1, 1, 0), (111, 1, 1, 1), (100, 0, 0, 1), (0, 0, 0, 0)):
        p = np.zeros(26, np.int32)
        p[4:8] = (iaer, sw, lw, vo)
        p[25] = 1
        f = driver._aer_flags(ctx(rad_physparam=p, aer_volc=SimpleNamespace(kyrsav=1991, kmonsav=6)))
        assert (f["iaerflg"], f["laswflg"], f["lalwflg"], f["lavoflg"]) == (iaer, bool(sw), bool(lw), bool(vo))
        assert (f["ivflip"], f["kyrsav"], f["kmonsav"]) == (1, 1991, 6)
    st = {"iaerflg": 11, "laswflg": True, "lalwflg": False, "lavoflg": False, "ivflip": 0, "kyrsav": 2, "kmonsav": 3}
    assert driver._aer_flags(ctx(aer_state=st, rad_physparam=np.zeros(26, np.int32))) is st
