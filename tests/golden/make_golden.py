"""Regenerate tests/golden/reference_ops.npz from the reference's own setup
numerics (oracle/_ref/libbfam_ref_ops.so, built from the reference source by
oracle/build_ref.sh).  Run in a checkout where the reference is present:

    bash oracle/build_ref.sh && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as orc  # noqa: E402


def main() -> None:
    out = {}
    for N in range(1, 9):
        r, w, wi, D = orc.ref_lgl(N)
        out[f"r_{N}"], out[f"w_{N}"], out[f"wi_{N}"], out[f"Dr_{N}"] = r, w, wi, D
        M = np.zeros((N + 1) ** 2)
        orc.ref_lib().bfam_ref_mass(N, M.ctypes.data_as(orc.dp))
        out[f"M_{N}"] = M
    for a, b in [(n, n) for n in range(1, 9)] + [(3, 5), (5, 3), (5, 7), (7, 5)]:
        prj, mp, wmp = orc.ref_interpolator(a, b)
        out[f"prj_{a}_to_{b}"] = prj
        out[f"massprj_{a}_to_{b}"] = mp
        out[f"wimassprj_{a}_to_{b}"] = wmp
    out["pcg32_0_1"] = orc.ref_pcg32(0, 1, 256)
    out["pcg32_42_54"] = orc.ref_pcg32(42, 54, 64)
    out["pcg32_1_2"] = orc.ref_pcg32(1, 2, 64)
    np.savez_compressed(Path(__file__).with_name("reference_ops.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
