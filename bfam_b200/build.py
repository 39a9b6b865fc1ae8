"""Build recipe for the in-tree shared libraries.

    python -m bfam_b200.build            # product library + oracle
    python -m bfam_b200.build --product  # product library only

Products:
  bfam_b200/libbfam_b200.so  -- CUDA kernels for sm_100a, the bfam_gpu C-ABI
                                and the host front end (mesher, operators)
  oracle/liboracle.so        -- the CPU oracle (test infrastructure)
  oracle/_ref/*               -- the reference compiled from its source
                                (oracle/build_ref.sh; only when
                                BFAM_REFERENCE_DIR is set)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "bfam_b200"
CSRC = PKG / "csrc"
LIB = PKG / "libbfam_b200.so"
ORACLE_LIB = ROOT / "oracle" / "liboracle.so"

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted((CSRC / "host").glob("*.c"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps)


def build_product(force: bool = False, verbose: bool = False) -> Path:
    headers = (sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h"))
               + sorted((ROOT / "include").glob("*.h")))
    deps = _sources() + headers
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    flags = [*NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17",
             "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
             "--expt-relaxed-constexpr",
             "-I", str(ROOT / "include"), "-I", str(CSRC)]
    if verbose:
        flags.insert(0, "-Xptxas=-v")

    def compile_one(src: Path) -> Path:
        obj = objdir / (src.name + ".o")
        if force or _stale(obj, [src] + headers):
            subprocess.run([_nvcc(), *flags, "-c", "-o", str(obj), str(src)], check=True)
        return obj

    # translation units compile in parallel (the kernel instantiations dominate)
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, _sources()))
    subprocess.run([_nvcc(), *NVCC_ARCH, "-shared", "-o", str(LIB), *map(str, objs)],
                   check=True)
    return LIB


def build_oracle(force: bool = False) -> Path:
    src = ROOT / "oracle" / "dg_oracle.c"
    if force or _stale(ORACLE_LIB, [src]):
        subprocess.run(
            ["gcc", "-std=gnu99", "-O2", "-fopenmp", "-fPIC", "-shared",
             "-o", str(ORACLE_LIB), str(src), "-lm"],
            check=True,
        )
    # the reference compiled from its own source (oracle/_ref), when
    # BFAM_REFERENCE_DIR names the reference checkout; otherwise the files
    # already in oracle/_ref are used as they are
    if os.environ.get("BFAM_REFERENCE_DIR"):
        subprocess.run(["bash", str(ROOT / "oracle" / "build_ref.sh")], check=True)
    return ORACLE_LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--product", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    build_product(force=a.force, verbose=a.verbose)
    if not a.product:
        build_oracle(force=a.force)
    return 0


if __name__ == "__main__":
    sys.exit(main())
