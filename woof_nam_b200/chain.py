"""One radiation call of a whole domain on one stream, without row windows: grrad's front end on the GPU
feeding the column solve.

The reference runs its radiation call (namgpu/physics/rrtm/rrtm_call.py:1-46) per window of rows, because
its chain's scratch for the whole domain does not fit its cards and its SW groups are per window
(rrtm_call.py:108-203).  Here every routine runs over all jm * im columns at once, in grrad_nmmb's order
(grrad_nmmb.f:660-2201):

    rad_grrad_setup   the radiation layers (plvl, plyr, tlyr, tlvl, qlyr, rhly, qstl, prslk1, tvly, tsfg)
    rad_dayparts      the SW interval's zenith cosine (coszen: the solve's day predicate) and the sunlit runs
    rad_getozn        olyr, climatological ozone on the layers (ntoz 0)
    rad_getgases      gasvmr on the layers
    rad_setaer        faersw, faerlw: the climatological aerosol optics (iaer 11), when an Aerosols is given
    rad_grrad_clw     clw from the cloud tracers, when ntcw is given
    rad_progcld2      clouds (Ferrier, np3d 3) with gethml's deck fractions
    rad_payne_albedo  the IALB = 2 albedos from sfcalbedo, sm and the daytime zenith cosine, with ialbflg 2
    rad_setalb        sfcalb (from coszen for ialbflg 0 / 1)
    rad_setemis       sfcemis
    rad_solve         LW and SW: heating rates and fluxes

about 8 launches ahead of the solve's own, no host synchronisation and no allocation once the work tensors
exist (pass the dict a previous call returned as `work`), so the whole call can be captured in one CUDA graph.

    from woof_nam_b200.chain import radiation_call
    out = radiation_call(solver, state, clim, sun=sun, solhr=12.0, dtswav=1200 / 3600, nrads=48, im=954)

`state` holds device tensors: the model state (pint [lm + 1][n], pmid, prslk, t, q [lm][n] in Pa / K / kg/kg,
tsfc [n]), the cloud fields on the lm + 1 radiation layers (clw, f_ice, f_rain, r_rime and, for a Thompson
cloud fraction, cldfk1), the grid (glon, glat, sinlat, coslat [n], radians) and the surface fields setalb and
setemis read (front.setalb / front.setemis names).  `clim` holds the CO2 and ozone climatologies (front.getgases /
front.getozn keyword arguments) and the emissivity map idxems.
"""
from __future__ import annotations

from . import _lib, front
from .grrad import layers as grrad_layers

CLOUD_NAM = dict(ivflip=0, llyr=2, iovr=1, lcrick=False, lcnorm=False, lnoprec=False, lsashal=False, cld_fraction=0)


def radiation_call(solver, state: dict, clim: dict, *, sun: dict, solhr: float, dtswav: float, nrads: int, im: int,
                   kmonsav: int, k1oz: int, k2oz: int, facoz: float, ico2flg: int = 1, ialbflg: int = 2,
                   iemslw: int = 1, cloud: dict | None = None, aerosols=None, ntcw: int | None = None,
                   ncld: int = 1, work: dict | None = None, out: dict | None = None, stream=None) -> dict:
    """Run the call; returns the solve's outputs, with the front end's arrays under out["work"] (reused by the
    next call when passed back as `work`).  aerosols: an aerosols.Aerosols with the month's climatology loaded
    (the state then needs slmsk), or None for no aerosol; state faersw / faerlw are used when given instead.
    ntcw (1-based): the condensate clw comes from the tracers state["tracer1"] [ntrac, lmk, n] (grrad's clw);
    else state["clw"] is read.  With ialbflg 2 and state["sfcalbedo"] (and "sm"), grrad's IALB = 2 block forms
    the albedos setalb reads from it and the daytime zenith cosine; else state's alvsf ... facwf are read."""
    cloud = {**CLOUD_NAM, **(cloud or {})}
    if cloud["ivflip"] != 0:
        raise ValueError("radiation_call: the layers of grrad's set-up are top first (ivflip 0)")
    torch = front._torch()
    n = state["tsfc"].numel()
    lm = state["pmid"].shape[0]
    lmk = lm + 1
    if solver.cfg.nlay != lmk:
        raise ValueError(f"radiation_call: the solver takes {solver.cfg.nlay} layers, the model state gives {lmk}")
    dev = state["tsfc"].device
    w = work or {}
    if not w:
        f32 = dict(dtype=torch.float32, device=dev)
        w["layers"] = None
        w["gasvmr"] = torch.empty((front.NF_VGAS, lmk, n), **f32)
        w["olyr"] = torch.zeros((lmk, n), **f32)
        w["sfcalb"] = torch.empty((front.NF_ALBD, n), **f32)
        w["sfcemis"] = torch.empty(n, **f32)
        w["dayparts"] = None
        w["cloud"] = None
    # grrad's layers, then the routines that read them, in grrad_nmmb's order
    w["layers"] = grrad_layers(solver, {k: state[k] for k in _lib.MODEL_FIELDS}, out=w["layers"], stream=stream)
    lay = w["layers"]
    w["dayparts"] = front.dayparts(solver, state["glon"], state["sinlat"], state["coslat"], solhr, dtswav, nrads, sun,
                                   im, out=w["dayparts"], stream=stream)
    coszen = w["dayparts"]["coszen"]
    front.getozn(solver, lay["prslk1"], state["glat"], w["olyr"], o3r=clim["o3r"], pkstr=clim["pkstr"], k1oz=k1oz,
                 k2oz=k2oz, facoz=facoz, blte=clim["blte"], dlte=clim["dlte"], ivflip=0, stream=stream)
    front.getgases(solver, lay["plvl"], state["glon"], state["glat"], w["gasvmr"], co2_glb=clim["co2_glb"],
                   gco2cyc=clim["gco2cyc"], co2vmr_sav=clim["co2vmr_sav"], ico2flg=ico2flg, kmonsav=kmonsav,
                   ivflip=0, stream=stream)
    if aerosols is not None:
        w["faer"] = aerosols.optics({k: lay[k] for k in ("plvl", "plyr", "tlyr", "qlyr")}, lay["rhly"], state["glon"],
                                    state["glat"], state["slmsk"], out=w.get("faer"), stream=stream)
    cin = {k: lay[k] for k in ("plyr", "plvl", "tlyr", "tvly", "qlyr", "qstl", "rhly")}
    cin.update({k: state.get(k) for k in ("clw", "f_ice", "f_rain", "r_rime", "cldfk1")}, xlat=state["glat"])
    if ntcw is not None:
        w["clw"] = front.grrad_clw(solver, state["tracer1"], ntcw, ncld, clw=w.get("clw"), stream=stream)
        cin["clw"] = w["clw"]
    w["cloud"] = front.progcld2(solver, cin, **cloud, out=w["cloud"], stream=stream)
    sfc = dict(state, coszf=coszen)
    if ialbflg == 2 and state.get("sfcalbedo") is not None:
        w["albedo"] = front.payne_albedo(solver, state["sfcalbedo"], state["sm"], coszen, out=w.get("albedo"),
                                         stream=stream)
        sfc.update({k: w["albedo"][k] for k in ("alvsf", "alnsf", "alvwf", "alnwf", "facsf", "facwf")})
    front.setalb(solver, sfc, ialbflg, w["sfcalb"], stream=stream)
    front.setemis(solver, state, clim.get("idxems"), ialbflg, iemslw, w["sfcemis"], stream=stream)
    cols = {"plyr": lay["plyr"], "plvl": lay["plvl"], "tlyr": lay["tlyr"], "tlvl": lay["tlvl"], "qlyr": lay["qlyr"],
            "olyr": w["olyr"], "gasvmr": w["gasvmr"], "clouds": w["cloud"]["clouds"], "sfcemis": w["sfcemis"],
            "tsfg": lay["tsfg"], "sfcalb": w["sfcalb"], "coszen": coszen}
    if aerosols is not None:
        cols["faersw"], cols["faerlw"] = w["faer"]
    for k in ("faerlw", "faersw"):
        if state.get(k) is not None:
            cols[k] = state[k]
    res = dict(solver.solve(cols, sun["solcon"], out=out, stream=stream))
    res["work"] = w
    return res
