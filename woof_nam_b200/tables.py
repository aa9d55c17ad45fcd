"""The packed RRTM tables as the library's table blob (rad_load_tables)."""
from __future__ import annotations

import struct
from functools import lru_cache
from pathlib import Path

import numpy as np

NPZ = Path(__file__).resolve().parent / "data" / "rrtm_tables.npz"


@lru_cache(maxsize=1)
def blob() -> bytes:
    """Serialise every table of rrtm_tables.npz: b"RADTBL01", uint32 count, then per table a uint16
    name length, the name, a uint8 dtype (0 float32, 1 float64, 2 int32), a uint64 element count and the
    little-endian data."""
    z = np.load(NPZ)
    parts = [b"RADTBL01", struct.pack("<I", len(z.files))]
    for name in z.files:
        a = z[name]
        if a.dtype.kind == "i":
            dt, b = 2, np.ascontiguousarray(a, dtype="<i4")
        elif a.dtype == np.float64:
            dt, b = 1, np.ascontiguousarray(a, dtype="<f8")
        else:
            dt, b = 0, np.ascontiguousarray(a, dtype="<f4")
        nb = name.encode()
        parts += [struct.pack("<H", len(nb)), nb, struct.pack("<BQ", dt, b.size), b.tobytes()]
    return b"".join(parts)
