"""Generate post_golden.npz: the reference's own rrtm_post_outputs kernel (namgpu/kernels/
phys_rrtm_driver_post.cu:71-145), compiled for the host into oracle/_ref/libref_rrtm.so by
oracle/build_ref.sh, on seeded inputs (oracle.post.make_case: 128 columns, 60 layers, a quarter of them
dry), on an LW step and on an SW-only step.

  in_*, state_*     the inputs and the accumulators before the call
  lw_*, sw_*        every output (and the updated cldcov / cldsa) with lw_step 1 and 0

Run from the repository root:  python tests/golden/make_post_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle, post  # noqa: E402

OUT = Path(__file__).resolve().parent / "post_golden.npz"
N, LM, SEED = 128, 60, 2024


def main():
    if not oracle.REF_LIB.exists():
        raise SystemExit("oracle/_ref/libref_rrtm.so is missing: run oracle/build_ref.sh first")
    inp, state = post.make_case(N, LM, SEED)
    blob = {f"in_{k}": v for k, v in inp.items()}
    blob.update({f"state_{k}": v for k, v in state.items()})
    for tag, lw in (("lw", True), ("sw", False)):
        r = post.reference_post(inp, state, LM, lw_step=lw)
        blob.update({f"{tag}_{k}": v for k, v in r.items()})
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
