"""Python front end of the B200 RRTM column radiation: device buffers in PyTorch, compute in libradb200.so.

``RadSolver`` mirrors the reference's column-solve entry (lwrad + swrad as ``rrtm_call`` drives them,
namgpu/physics/rrtm/rrtm_call.py:246): it takes the radiation driver's column state in the reference's
layout and returns the LW/SW heating rates and the surface and TOA fluxes under the reference's names.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace

import numpy as np

from . import _lib
from .tables import blob

INPUT_FIELDS = ("plyr", "plvl", "tlyr", "tlvl", "qlyr", "olyr", "gasvmr", "clouds", "sfcemis", "tsfg",
                "sfcalb", "coszen")
# inputs each solve reads (lwrad / swrad argument lists, phys_rrtm_lw_lwrad.py:36-46, phys_rrtm_sw_swrad.py:34-43)
PART_FIELDS = {"lw": ("plyr", "plvl", "tlyr", "tlvl", "qlyr", "olyr", "gasvmr", "clouds", "sfcemis", "tsfg"),
               "sw": ("plyr", "plvl", "tlyr", "qlyr", "olyr", "gasvmr", "clouds", "sfcalb", "coszen"),
               "both": INPUT_FIELDS}
OPTIONAL_INPUTS = ("faerlw", "faersw", "icseed")


def _torch():
    import torch
    return torch


@dataclass
class SolverConfig:
    nlay: int = 61
    precision: str = "mixed"         # "mixed" or "fp64"
    route: str = "nam"               # "nam" (rtrnmr + spcvrtc) or "mcica"
    iswmode: int = 2                 # 1 delta-Eddington, 2 PIFM (NAM), 3 discrete ordinates
    diagnostic: bool = False         # clouds give optical depth / SSA / asymmetry directly
    window_cols: int = 0             # SW MINVAL(laytrop) window in columns (0 = whole request)
    sw_chunk: int = 32768
    cpathfac: float = 1.5
    iovrlw: int = 1                  # cloud overlap, 0 random, 1 maximum-random, 2 maximum: McICA generators;
    iovrsw: int = 1                  # on the NAM route iovrlw 0 = rtrn (else rtrnmr), iovrsw = swrad's zcf0
    lw_seed0: int = 140              # McICA seed offsets (ipsdlw0, ipsdsw0)
    sw_seed0: int = 1
    parts: str = "both"              # "lw", "sw" or "both": which solves run (lslwr / lsswr steps)
    lw_chunk: int = 0                # mixed: columns per two-kernel LW chunk (0 = 32768, < 0 single kernel)
    sw_sweep_chunk: int = 0          # mixed: day columns per two-kernel SW chunk (0 = 16384, < 0 single kernel)
    # optional outputs of lwrad / swrad (the reference's lhlw0, lhlwb, lhsw0, lhswb / has_htrswb, lflxprf switches)
    lhlw0: bool = False              # hlw0 [nlay][ncol]: LW clear-sky heating
    lhlwb: bool = False              # hlwb [16][nlay][ncol]: LW heating per band
    lhsw0: bool = False              # hsw0 [nlay][ncol]: SW clear-sky heating
    lhswb: bool = False              # htswb [14][nlay][ncol]: SW heating per band
    lflxprf: bool = False            # lwflxprf / swflxprf [4][nlay + 1][ncol]: level fluxes


OPTIONAL_OUTPUTS = ("hsw0", "htswb", "swflxprf", "hlw0", "hlwb", "lwflxprf")


def output_shapes(nlay: int, ncol: int, route: str = "nam", cfg: "SolverConfig | None" = None) -> dict:
    """Output arrays of a solve; the McICA route adds the sub-column cloud words (int32 storage of the
    uint32 words, [word][layer][column], layers surface first, bit g & 31 of word g >> 5); cfg's switches add
    the optional outputs (levels top first)."""
    d = {"htlw": (nlay, ncol), "htsw": (nlay, ncol), "topflw": (2, ncol), "sfcflw": (4, ncol),
         "topfsw": (3, ncol), "sfcfsw": (4, ncol), "fdncmp": (6, ncol)}
    if route == "mcica":
        d["lw_mask"] = (5, nlay, ncol)
        d["sw_mask"] = (4, nlay, ncol)
    if cfg is not None:
        if cfg.lhsw0:
            d["hsw0"] = (nlay, ncol)
        if cfg.lhswb:
            d["htswb"] = (14, nlay, ncol)
        if cfg.lhlw0:
            d["hlw0"] = (nlay, ncol)
        if cfg.lhlwb:
            d["hlwb"] = (16, nlay, ncol)
        if cfg.lflxprf:
            d["swflxprf"] = (4, nlay + 1, ncol)
            d["lwflxprf"] = (4, nlay + 1, ncol)
    return d


MASK_KEYS = ("lw_mask", "sw_mask")


def _fits(t, shape: tuple) -> bool:
    """t holds exactly the elements of `shape` with the columns last (a [3][14][nlay][ncol] array may come as
    [42][nlay][ncol]: the kernels read contiguous memory by nlay and ncol alone)."""
    return t.dim() >= 1 and t.shape[-1] == shape[-1] and t.numel() == int(np.prod(shape))


def input_shapes(nlay: int, ncol: int) -> dict:
    """Shapes of a solve's inputs (RadColumns), the optional ones included."""
    return {"plyr": (nlay, ncol), "plvl": (nlay + 1, ncol), "tlyr": (nlay, ncol), "tlvl": (nlay + 1, ncol),
            "qlyr": (nlay, ncol), "olyr": (nlay, ncol), "gasvmr": (10, nlay, ncol), "clouds": (9, nlay, ncol),
            "faerlw": (3, 16, nlay, ncol), "faersw": (3, 14, nlay, ncol), "sfcemis": (ncol,), "tsfg": (ncol,),
            "sfcalb": (4, ncol), "coszen": (ncol,), "icseed": (2, ncol)}


class RadSolver:
    """One library handle on the current CUDA device."""

    def __init__(self, cfg: SolverConfig | None = None, **kw):
        self.cfg = cfg or SolverConfig(**kw)
        self.lib = _lib.load()
        c = _lib.RadConfig()
        self.lib.rad_config_default(ctypes.byref(c), self.cfg.nlay)
        c.precision = _lib.PREC[self.cfg.precision]
        c.route = _lib.ROUTE[self.cfg.route]
        c.iswmode = self.cfg.iswmode
        c.diagnostic = int(self.cfg.diagnostic)
        c.window_cols = self.cfg.window_cols
        c.sw_chunk = self.cfg.sw_chunk
        c.cpathfac = self.cfg.cpathfac
        c.parts = _lib.PARTS[self.cfg.parts]
        c.lw_chunk = self.cfg.lw_chunk
        c.sw_sweep_chunk = self.cfg.sw_sweep_chunk
        c.iovrlw, c.iovrsw = self.cfg.iovrlw, self.cfg.iovrsw
        c.lw_seed0, c.sw_seed0 = self.cfg.lw_seed0, self.cfg.sw_seed0
        h = ctypes.c_void_p()
        _lib.check(self.lib, None, self.lib.rad_create(ctypes.byref(c), ctypes.byref(h)), "rad_create")
        self.handle = h
        b = blob()
        _lib.check(self.lib, h, self.lib.rad_load_tables(h, b, len(b)), "rad_load_tables")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.rad_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------------------------------------
    def alloc_outputs(self, ncol: int, device=None) -> dict:
        """Output tensors of a solve of ncol columns (those of the configured parts only)."""
        torch = _torch()
        skip = {"lw": ("htsw", "topfsw", "sfcfsw", "fdncmp", "hsw0", "htswb", "swflxprf"),
                "sw": ("htlw", "topflw", "sfcflw", "hlw0", "hlwb", "lwflxprf"), "both": ()}[self.cfg.parts]
        return {k: torch.empty(s, dtype=torch.int32 if k in MASK_KEYS else torch.float32, device=device or "cuda")
                for k, s in output_shapes(self.cfg.nlay, ncol, self.cfg.route, self.cfg).items() if k not in skip}

    def _abi_args(self, cols: dict, solcon: float, out: dict | None):
        torch = _torch()
        ncol = int(cols["plyr"].shape[-1])
        # shapes first (the kernels index by nlay and ncol alone), then devices and types
        if cols["plyr"].shape[0] != self.cfg.nlay:
            raise ValueError(f"plyr has {cols['plyr'].shape[0]} layers, the solver was built for {self.cfg.nlay}")
        want = input_shapes(self.cfg.nlay, ncol)
        for k in PART_FIELDS[self.cfg.parts]:
            if cols.get(k) is None:
                raise KeyError(f"input {k!r} is missing")
        for k, shp in want.items():
            t = cols.get(k)
            if t is not None and not _fits(t, shp):
                raise ValueError(f"input {k!r} has shape {tuple(t.shape)}, expected {shp} (or the same elements with "
                                 "the columns last)")
        for k in PART_FIELDS[self.cfg.parts]:
            t = cols[k]
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                raise TypeError(f"input {k!r} must be a contiguous float32 CUDA tensor")
        if out is None:
            out = self.alloc_outputs(ncol, device=cols["plyr"].device)
        ci = _lib.RadColumns()
        for k in INPUT_FIELDS:
            t = cols.get(k)
            setattr(ci, k, t.data_ptr() if t is not None else None)
        for k in OPTIONAL_INPUTS:
            t = cols.get(k)
            if t is not None:
                want = torch.int32 if k == "icseed" else torch.float32
                if not (t.is_cuda and t.dtype == want and t.is_contiguous()):
                    raise TypeError(f"input {k!r} must be a contiguous {want} CUDA tensor")
            setattr(ci, k, t.data_ptr() if t is not None else None)
        ci.solcon = float(solcon)
        co = _lib.RadOutputs()
        full = output_shapes(self.cfg.nlay, ncol, "mcica", replace(self.cfg, lhsw0=True, lhswb=True, lhlw0=True,
                                                                   lhlwb=True, lflxprf=True))
        for k in tuple(output_shapes(1, 1, "mcica")) + OPTIONAL_OUTPUTS:
            t = out.get(k)
            if t is not None:
                dt = torch.int32 if k in MASK_KEYS else torch.float32
                if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dt and t.is_contiguous()):
                    raise TypeError(f"output {k!r} must be a contiguous {dt} CUDA tensor")
                if not _fits(t, full[k]):
                    raise ValueError(f"output {k!r} has shape {tuple(t.shape)}, expected {full[k]}")
            setattr(co, k, t.data_ptr() if t is not None else None)
        return ci, co, ncol, out

    def solve(self, cols: dict, solcon: float, out: dict | None = None, stream=None) -> dict:
        """Solve device-resident columns.  ``cols`` maps the reference names (INPUT_FIELDS, optionally
        faerlw/faersw/icseed) to contiguous float32 CUDA tensors in [field][level][column] layout."""
        torch = _torch()
        ci, co, ncol, out = self._abi_args(cols, solcon, out)
        st = stream if stream is not None else torch.cuda.current_stream()
        rc = self.lib.rad_solve(self.handle, ctypes.byref(ci), ctypes.byref(co), ncol, ctypes.c_void_p(st.cuda_stream))
        _lib.check(self.lib, self.handle, rc, "rad_solve")
        return out

    def solve_batch(self, requests: list, solcons: list, outs: list | None = None, stream=None) -> list:
        """Several independent requests in one call (rad_solve_batch); each keeps its own SW groups."""
        torch = _torch()
        n = len(requests)
        outs = outs or [None] * n
        args = [self._abi_args(c, s, o) for c, s, o in zip(requests, solcons, outs)]
        ins = (_lib.RadColumns * max(n, 1))(*[a[0] for a in args])
        ous = (_lib.RadOutputs * max(n, 1))(*[a[1] for a in args])
        ncols = (ctypes.c_int64 * max(n, 1))(*[a[2] for a in args])
        st = stream if stream is not None else torch.cuda.current_stream()
        rc = self.lib.rad_solve_batch(self.handle, n, ins, ous, ncols, ctypes.c_void_p(st.cuda_stream))
        _lib.check(self.lib, self.handle, rc, "rad_solve_batch")
        return [a[3] for a in args]

    def to_device(self, columns, device="cuda", pinned: bool = False, icseed=None) -> dict:
        """Copy a woof_nam_b200.columns.Columns request to the device (optionally through pinned memory).
        icseed: optional McICA seeds, int32 [2][ncol] (LW row, SW row)."""
        torch = _torch()
        d = {}
        for k in INPUT_FIELDS:
            a = torch.from_numpy(np.ascontiguousarray(getattr(columns, k), dtype=np.float32))
            if pinned:
                a = a.pin_memory()
            d[k] = a.to(device, non_blocking=pinned)
        if icseed is not None:
            d["icseed"] = torch.from_numpy(np.ascontiguousarray(icseed, dtype=np.int32)).to(device)
        return d

    def solve_host(self, columns, icseed=None) -> dict:
        """Host arrays in, host arrays out (copies both ways)."""
        torch = _torch()
        d = self.to_device(columns, icseed=icseed)
        out = self.solve(d, columns.solcon)
        torch.cuda.synchronize()
        r = {k: v.cpu().numpy() for k, v in out.items()}
        for k in MASK_KEYS:
            if k in r:
                r[k] = r[k].view(np.uint32)
        return r

    def capture(self, requests: list, solcons: list, outs: list | None = None) -> "SolveGraph":
        """Capture a batched solve of device-resident requests into a CUDA graph (rad_graph_create).  The
        graph keeps the tensors' addresses: refill the inputs in place and replay with SolveGraph.launch()."""
        n = len(requests)
        outs = outs or [None] * n
        args = [self._abi_args(c, s, o) for c, s, o in zip(requests, solcons, outs)]
        ins = (_lib.RadColumns * max(n, 1))(*[a[0] for a in args])
        ous = (_lib.RadOutputs * max(n, 1))(*[a[1] for a in args])
        ncols = (ctypes.c_int64 * max(n, 1))(*[a[2] for a in args])
        g = ctypes.c_void_p()
        _lib.check(self.lib, self.handle, self.lib.rad_graph_create(self.handle, n, ins, ous, ncols, ctypes.byref(g)),
                   "rad_graph_create")
        return SolveGraph(self, g, requests, [a[3] for a in args])

    def post_outputs(self, inp: dict, out: dict, lm: int, kd: int = 1, cloud_block: bool = True,
                     lw_step: bool = True, stream=None) -> dict:
        """The radiation call's post step (rad_post_outputs; rrtm_post_outputs of the reference,
        phys_rrtm_driver_post.cu:71-145): inp / out map the lower-case names of RadPostIn / RadPostOut to
        contiguous CUDA tensors ([level or component][ncol]; cu_cloud, ncfrst, ncfrcv int32).  With kd = 1,
        hlw / swh are the solve's [nlay] htlw / htsw."""
        torch = _torch()
        n = int(inp["coszen_v"].shape[-1])
        pi, po = _lib.RadPostIn(), _lib.RadPostOut()
        for k in _lib.POST_IN_FIELDS:
            t = inp.get(k)
            if t is not None and not (t.is_cuda and t.is_contiguous() and t.shape[-1] == n):
                raise TypeError(f"post input {k!r} must be a contiguous CUDA tensor with {n} columns")
            setattr(pi, k, t.data_ptr() if t is not None else None)
        for k in _lib.POST_OUT_FIELDS:
            t = out.get(k)
            if t is not None and not (t.is_cuda and t.is_contiguous() and t.shape[-1] == n):
                raise TypeError(f"post output {k!r} must be a contiguous CUDA tensor with {n} columns")
            setattr(po, k, t.data_ptr() if t is not None else None)
        st = stream if stream is not None else torch.cuda.current_stream()
        rc = self.lib.rad_post_outputs(self.handle, ctypes.byref(pi), ctypes.byref(po), n, lm, kd, int(cloud_block),
                                       int(lw_step), ctypes.c_void_p(st.cuda_stream))
        _lib.check(self.lib, self.handle, rc, "rad_post_outputs")
        return out

    def rdtemp(self, p: dict, stream=None) -> None:
        """RDTEMP on the device (rad_rdtemp; rdtemp_apply of the reference, drv_rdtemp.cu:140-198): p holds
        the scalars of RadRdtemp and the CUDA tensors glat, glon, czmean ([jm, im]), rswtt, rlwtt, t
        ([lm, jm, im]) and czen ([jm, im]); t and czen are updated in place."""
        torch = _torch()
        r = _lib.RadRdtemp()
        for k, _ in r._fields_:
            v = p[k]
            if isinstance(v, torch.Tensor):
                if not (v.is_cuda and v.dtype == torch.float32 and v.is_contiguous()):
                    raise TypeError(f"rdtemp: {k} must be a contiguous float32 CUDA tensor")
                setattr(r, k, v.data_ptr())
            else:
                setattr(r, k, v)
        st = stream if stream is not None else torch.cuda.current_stream()
        _lib.check(self.lib, self.handle, self.lib.rad_rdtemp(self.handle, ctypes.byref(r), ctypes.c_void_p(st.cuda_stream)),
                   "rad_rdtemp")

    def device_error(self) -> int:
        """The device error word since the last call (0: none; see rad_device_error), then cleared."""
        code = ctypes.c_int32()
        rc = self.lib.rad_device_error(self.handle, ctypes.byref(code))
        _lib.check(self.lib, self.handle, rc, "rad_device_error")
        return int(code.value)

    def profile(self, on: bool = True) -> None:
        """Start (or stop) device-time accounting of the library's kernels on this handle."""
        _lib.check(self.lib, self.handle, self.lib.rad_profile_enable(self.handle, int(on)), "rad_profile_enable")

    def profile_read(self) -> dict:
        """Kernel launches since creation and device ms of the LW / SW-prep / SW kernels since profile()."""
        p = _lib.RadProfile()
        _lib.check(self.lib, self.handle, self.lib.rad_profile_read(self.handle, ctypes.byref(p)), "rad_profile_read")
        return {k: getattr(p, k) for k, _ in p._fields_}

    def workspace_bytes(self, ncol: int) -> int:
        return int(self.lib.rad_workspace_bytes(self.handle, ncol))


class SolveGraph:
    """A captured batched solve; holds references to its tensors so their memory outlives the graph."""

    def __init__(self, solver: RadSolver, g, requests, outs):
        self.solver, self.g, self.requests, self.outs = solver, g, requests, outs

    def launch(self, stream=None) -> list:
        torch = _torch()
        st = stream if stream is not None else torch.cuda.current_stream()
        _lib.check(self.solver.lib, self.solver.handle, self.solver.lib.rad_graph_launch(self.g, ctypes.c_void_p(st.cuda_stream)),
                   "rad_graph_launch")
        return self.outs

    def close(self):
        if getattr(self, "g", None):
            self.solver.lib.rad_graph_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
