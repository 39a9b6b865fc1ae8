"""Shared-memory face-array layout of the stage kernel, checked on the host.

At 3D N=7 the face arrays (neighbour traces, flux jumps, mortar jumps) are
stored with rows and columns XOR-swizzled by array index (`fpos` in
`bfam_b200/csrc/dg_common.cuh`).  `tests/c/face_layout_check.cu` calls the
same inline functions the kernel uses (compiled for the host by nvcc) and
checks that each array's positions are a permutation of its slots (no two
face nodes share a slot) and that the mortar line passes and the face-node
passes meet 16 distinct bank pairs per half-warp.  No GPU is needed.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("nvcc") is None and not Path("/usr/local/cuda/bin/nvcc").exists(),
                    reason="nvcc not available")
def test_face_layout_permutation_and_banks(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "face_layout_check"
    subprocess.run(
        # PTX-only device target: the check runs on the host, so ptxas is
        # not needed
        [nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=compute_100a",
         "--expt-relaxed-constexpr", "-I", str(ROOT / "bfam_b200" / "csrc"),
         "-I", str(ROOT / "include"), "-o", str(exe),
         str(ROOT / "tests" / "c" / "face_layout_check.cu")],
        check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
