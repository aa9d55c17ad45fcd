"""Pack the climatological aerosol data of the NAM radiation (OPAC, 5-degree global) into aer_tables.npz.

Runs where the reference tree is available and writes ``aer_tables.npz`` next to this script; the library,
the oracle and the tests load the packed file, nothing at run time reads the reference tree.  Sources:

* ``namgpu/parm/nam_climaeropac_global.txt`` -- twelve monthly distributions (per 5-degree cell: up to five
  component indices with mixing ratios, the profile type, the number density), then the optical tables
  (ending wavenumbers of the 61 OPAC bands, scale heights and reference pressures of the 7 profile
  structures x 5 domains, extinction / scattering / single-scattering albedo / asymmetry of the 6
  humidity-independent species and of the 4 humidity-dependent species at 8 humidity levels, and the
  stratospheric background extinction).  Fixed-width records as the Fortran formats lay them out
  (monthly: 5 x (i2, e11.4), i2, f8.2; optical: 13i6, 20f4.1, 10f7.2, 8e10.3).
* the solar spectrum of set_spectrum -- 151 intervals (wavenumber count, flux per wavenumber), the DATA
  statements of radiation_aerosols_nmmb.f:166-215 as the reference carries them in
  ``namgpu/kernels/phys_rrtm_aer_init.cu`` (AER_NWVNS0, AER_S0INTV).

Numbers are stored as parsed: decimal text -> float64 -> float32 for the single-precision tables, float64
for the monthly mixing ratios and densities (the reference's aer_update keeps those in kind_phys double).

Usage:  python woof_nam_b200/data/pack_aer_tables.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np

IMXAE, JMXAE, NXC = 72, 37, 5
NAERBND, NRHLEV, NCM1, NCM2, NDM, NAE = 61, 8, 6, 4, 5, 7
MONTH_LINES = 2 + IMXAE * JMXAE


def _num(s: str) -> float:
    s = s.strip()
    if not s:
        return 0.0
    try:
        return float(s)
    except ValueError:           # Fortran E input without the exponent letter (1.0-10)
        k = max(s.rfind("+"), s.rfind("-"))
        return float(s[:k] + "E" + s[k:])


def _fields(lines, pos, n, per_line, width, conv):
    """A header line, then n values in fixed-width fields, per_line to a line.  Returns (next pos, values)."""
    pos += 1
    out = []
    while len(out) < n:
        ln = lines[pos]
        pos += 1
        for j in range(min(per_line, n - len(out))):
            out.append(conv(ln[j * width:(j + 1) * width]))
    return pos, out


def parse(path: Path) -> dict:
    lines = path.read_text().splitlines()
    t = {}
    idx = np.zeros((12, JMXAE, IMXAE, NXC), np.int8)
    cmix = np.zeros((12, JMXAE, IMXAE, NXC), np.float64)
    kprf = np.zeros((12, JMXAE, IMXAE), np.int8)
    denn = np.zeros((12, JMXAE, IMXAE), np.float64)
    for m in range(12):
        base = m * MONTH_LINES
        if "MONTH OF" not in lines[base]:
            raise RuntimeError(f"{path}: month {m + 1} header not at line {base + 1}")
        for r in range(JMXAE * IMXAE):
            ln = lines[base + 2 + r]
            j, i = divmod(r, IMXAE)               # records run latitude-major, longitude inner
            for k in range(NXC):
                idx[m, j, i, k] = int(ln[13 * k:13 * k + 2])
                cmix[m, j, i, k] = float(ln[13 * k + 2:13 * k + 13])
            kprf[m, j, i] = int(ln[65:67])
            denn[m, j, i] = float(ln[67:75])
    t.update(month_idx=idx, month_cmix=cmix, month_kprf=kprf, month_denn=denn)
    pos = 12 * MONTH_LINES
    if not lines[pos].startswith("ENDING WAVENUMBER"):
        raise RuntimeError(f"{path}: optical tables not at line {pos + 1}")
    pos, v = _fields(lines, pos, NAERBND, 13, 6, int)
    t["iendwv"] = np.array(v, np.int32)
    pos, v = _fields(lines, pos, NAE * NDM, 20, 4, _num)
    t["haer"] = np.array(v, np.float64).astype(np.float32).reshape(NAE, NDM)
    pos, v = _fields(lines, pos, NAE * NDM, 10, 7, _num)
    t["prsref"] = np.array(v, np.float64).astype(np.float32).reshape(NAE, NDM)
    for name in ("rhidext0", "rhidsca0", "rhidssa0", "rhidasy0"):
        pos, v = _fields(lines, pos, NAERBND * NCM1, 8, 10, _num)
        t[name] = np.array(v, np.float64).astype(np.float32).reshape(NCM1, NAERBND)
    for name in ("rhdpext0", "rhdpsca0", "rhdpssa0", "rhdpasy0"):
        pos, v = _fields(lines, pos, NAERBND * NRHLEV * NCM2, 8, 10, _num)
        t[name] = np.array(v, np.float64).astype(np.float32).reshape(NCM2, NRHLEV, NAERBND)
    if not lines[pos].startswith("STRATOSPERIC"):
        raise RuntimeError(f"{path}: stratospheric table not at line {pos + 1}")
    pos, v = _fields(lines, pos, NAERBND, 8, 10, _num)
    t["straext0"] = np.array(v, np.float64).astype(np.float32)
    return t


def solar_spectrum(cu: Path) -> dict:
    src = cu.read_text()
    def arr(name):
        m = re.search(name + r"\[[A-Z]+\]\s*=\s*\{([^}]*)\}", src)
        if not m:
            raise RuntimeError(f"{cu}: {name} not found")
        return [s.strip().rstrip("f") for s in m.group(1).split(",") if s.strip()]
    nw = np.array([int(s) for s in arr("AER_NWVNS0")], np.int32)
    s0 = np.array([float(s) for s in arr("AER_S0INTV")], np.float64).astype(np.float32)
    if nw.size != 151 or s0.size != 151 or int(nw.sum()) != 57600:
        raise RuntimeError("solar spectrum: expected 151 intervals over 57,600 wavenumbers")
    return {"nwvns0": nw, "s0intv": s0}


def main():
    if len(sys.argv) < 2:
        raise SystemExit("usage: python pack_aer_tables.py <reference tree>")
    root = Path(sys.argv[1])
    t = parse(root / "namgpu" / "parm" / "nam_climaeropac_global.txt")
    t.update(solar_spectrum(root / "namgpu" / "kernels" / "phys_rrtm_aer_init.cu"))
    out = Path(__file__).resolve().parent / "aer_tables.npz"
    np.savez_compressed(out, **t)
    print(f"wrote {out} ({out.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
