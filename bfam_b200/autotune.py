"""Tile autotuner for batches.

A batch runs one launch per order group, level and LSRK stage.  The tile of a
group is (elements per CTA, threads per element, register budget for a
number of resident CTAs per SM), chosen among the shapes compiled for that
order (`tile_shapes`, `tile_elements`), plus the CTAs per SM of a persistent
grid (two-buffer tiles) or of the L2 lookahead distance (one-buffer tiles).  The tuner times
every candidate on a synthetic domain of the group's order, precision and
roughly its element count (a 20 % refined brick, Gaussian pulse, random
material, capped in size so tuning takes seconds), with CUDA events on the
batch's stream over a few graph-replayed steps, and keeps the fastest.
Results are cached per GPU name in a JSON file.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

import numpy as np

from . import (Batch, BfamGpuError, GpuDomain, Mesh, lgl_operators, material_random,
               tile_elements, tile_shapes)

DEFAULT_CACHE = Path(__file__).resolve().parent / "tile_cache.json"
MAX_TUNE_ELEMENTS = 24000


def _brick_for(dim: int, elements: int, refine_prob: float = 0.2):
    """base cells per axis so that the refined brick has about `elements`"""
    base = max(1.0, elements / (1 + (2 ** dim - 1) * refine_prob))
    n = max(1, round(base ** (1.0 / dim)))
    return (n,) * dim


def _key(gpu: str, dim: int, N: int, precision: int) -> str:
    """cache key: the GPU, the group, and the library's tile table for the
    order (threads x register budget x elements per CTA of every tile), so
    that a library with another table never reuses a tile index chosen
    against the old one"""
    table = "-".join(f"{t}x{m}x{e}" for (t, m), e in
                     zip(tile_shapes(dim, N), tile_elements(dim, N)))
    return f"{gpu}|dim{dim}|N{N}|prec{precision}|tiles:{table}"


def load_cache(path: Path | None = None) -> dict:
    path = Path(path or os.environ.get("BFAM_B200_TILE_CACHE", DEFAULT_CACHE))
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: Path | None = None) -> None:
    path = Path(path or os.environ.get("BFAM_B200_TILE_CACHE", DEFAULT_CACHE))
    path.write_text(json.dumps(cache, indent=1, sort_keys=True) + "\n")


def tune_group(dim: int, N: int, precision: int, elements: int, steps: int = 4,
               device: int = 0, seed: int = 5) -> dict:
    """Time every (tile, CTAs per SM) candidate; returns the table and the best."""
    import torch

    n = _brick_for(dim, min(elements, MAX_TUNE_ELEMENTS))
    mesh = Mesh(dim, N, n, refine_prob=0.2, seed=seed)
    rho, lam, mu = material_random(mesh.K, seed)
    r = lgl_operators(N)[0]
    q0 = mesh.gaussian_pulse(r, (0.5, 0.5, 0.5), 0.1)
    cp = np.sqrt((lam + 2 * mu) / rho)
    dt = 0.3 * float(np.min(mesh.h[:, :dim].min(axis=1) / cp)) / (N * N)
    dom = GpuDomain(mesh, rho, lam, mu, precision=precision, device=device)
    dom.set_fields(q0)
    stream = torch.cuda.Stream(device=device)
    b = Batch([dom])
    b.set_stream(stream.cuda_stream)
    table = []
    shapes = tile_shapes(dim, N)
    epcs = tile_elements(dim, N)
    for tile, ((threads, minb), epc) in enumerate(zip(shapes, epcs)):
        for cps in sorted({0, max(1, minb - 1)} if minb > 1 else {0}):
            try:
                b.set_tile(0, tile, cps)
            except BfamGpuError:
                continue  # does not fit an SM on this device
            b.step([dt], 1)  # capture + warm-up
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.step([dt], steps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            table.append({"tile": tile, "threads": threads, "elements_per_cta": epc,
                          "min_ctas": minb, "ctas_per_sm": cps, "ms_per_step": ms,
                          "dof_updates_per_s": mesh.ndof * 5 / (ms / 1e3)})
    b.free()
    dom.free()
    best = min(table, key=lambda t: t["ms_per_step"])
    return {"best": {"tile": best["tile"], "ctas_per_sm": best["ctas_per_sm"]},
            "elements": mesh.K, "table": table}


def autotune(batch: Batch, cache: dict | None = None, cache_path=None,
             device: int = 0, save: bool = True) -> list[dict]:
    """Choose every group's tile of `batch` (from the cache, else by timing)
    and apply it.  Returns the choice per group."""
    import torch

    gpu = torch.cuda.get_device_name(device)
    own_cache = cache is None
    cache = load_cache(cache_path) if own_cache else cache
    choices = []
    dirty = False
    for g, info in enumerate(batch.groups()):
        key = _key(gpu, info["dim"], info["N"], info["precision"])
        if key not in cache:
            cache[key] = tune_group(info["dim"], info["N"], info["precision"],
                                    info["elements"], device=device)
            dirty = True
        best = cache[key]["best"]
        batch.set_tile(g, best["tile"], best["ctas_per_sm"])
        choices.append(dict(info, **best, table=cache[key].get("table", [])))
    if dirty and save and own_cache:
        save_cache(cache, cache_path)
    return choices
