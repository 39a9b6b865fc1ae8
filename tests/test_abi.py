"""The C-ABI library loads, exports every declared symbol, and rejects
malformed bfam arrays before touching the device."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import bfam_b200 as bf

INCLUDE = Path(__file__).resolve().parent.parent / "include"


# header-only: static inline functions over the exported C-ABI, compiled by
# the application against its own bfam.h
ADAPTER = "bfam_gpu_bfam.h"


def _code(h: Path) -> str:
    text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def declared_functions():
    names = []
    for h in sorted(INCLUDE.glob("*.h")):
        if h.name == ADAPTER:
            continue
        for m in re.finditer(r"\b(bfam_[A-Za-z0-9_]+)\s*\(", _code(h)):
            names.append(m.group(1))
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(str(bf.LIB_PATH))
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_adapter_calls_only_exported_entry_points():
    """The bfam adapter is header-only: every bfam_gpu_* / bfam_ts_lsrk_*
    function it calls and does not define inline is exported."""
    code = _code(INCLUDE / ADAPTER)
    inline = set(re.findall(r"static inline \w+\s*\*?\s*(bfam_\w+)\s*\(", code))
    called = set(re.findall(r"\b(bfam_(?:gpu|ts_lsrk)_\w+)\s*\(", code))
    lib = C.CDLL(str(bf.LIB_PATH))
    need = sorted(n for n in called - inline if not n.endswith("_t"))
    assert "bfam_gpu_domain_create_from_quadrants" in need
    missing = [n for n in need if not hasattr(lib, n)]
    assert not missing, missing
    assert {"bfam_gpu_domain_upload", "bfam_gpu_domain_upload_pxest",
            "bfam_gpu_domain_download", "bfam_gpu_lsrk_init"} <= inline


def test_rejects_rotated_tree_pairings():
    """The element metric is diagonal (aligned trees): a face meeting its
    neighbour's face with permuted nodes, a face meeting a non-opposite face
    and a glue element with a non-zero orientation are refused as
    unsupported, before any device call."""
    m = bf.Mesh(3, 2, (3, 3, 3))
    keep = []
    Nfp, NF, Np = m.Nfp, m.Nfaces, m.Np
    e, f = 4, 1
    sl = slice((e * NF + f) * Nfp, (e * NF + f + 1) * Nfp)
    nb = int(m.vmapP[sl][0]) // Np
    # the same neighbour face with its nodes transposed (orientation 1)
    perm = m.vmapP.copy()
    nodes = perm[sl].reshape(m.Nq, m.Nq)
    perm[sl] = nodes.T.reshape(-1)
    v = _vol(m, keep)
    v.vmapP = perm.ctypes.data_as(bf.i32p)
    keep.append(perm)
    rc, _ = _create(v)
    assert rc == bf.BFAM_GPU_EUNSUPPORTED and "permuted" in bf.last_error()
    # face f meeting the neighbour's face f (not f ^ 1)
    other = m.vmapP.copy()
    other[sl] = m.vmapM[(nb * NF + f) * Nfp:(nb * NF + f + 1) * Nfp]
    v = _vol(m, keep)
    v.vmapP = other.ctypes.data_as(bf.i32p)
    keep.append(other)
    rc, _ = _create(v)
    assert rc == bf.BFAM_GPU_EUNSUPPORTED and "aligned trees" in bf.last_error()
    # a glue element with orientation 3
    mg = bf.Mesh(3, 2, (2, 2, 2), refine_prob=0.5, seed=1)
    v = _vol(mg, keep)
    ops = bf.mortar_operators(2, 2)
    g = bf.GlueDesc()
    op = mg.EToOp.copy()
    op[0] = 3
    keep += [op, ops]
    g.K = mg.Kg
    g.EToEp = mg.EToEp.ctypes.data_as(bf.i32p)
    g.EToEm = mg.EToEm.ctypes.data_as(bf.i32p)
    for name in ("EToHp", "EToFm", "EToHm"):
        setattr(g, name, getattr(mg, name).ctypes.data_as(bf.i8p))
    g.EToOp = op.ctypes.data_as(bf.i8p)
    for s_, k in enumerate((0, 3, 4)):
        g.interpolation[s_] = bf._dp(ops[k]) if k else bf.dp()
    for s_, k in enumerate((0, 1, 2)):
        g.projection[s_] = bf._dp(ops[k]) if k else bf.dp()
    rc, _ = _create(v, g)
    assert rc == bf.BFAM_GPU_EUNSUPPORTED and "orientation 3" in bf.last_error()


def _vol(m, ops_keep):
    r, w, wi, D = bf.lgl_operators(m.N)
    rho, lam, mu = (np.ones(m.K), np.full(m.K, 2.0), np.ones(m.K))
    keep = [r, w, D, rho, lam, mu, np.ascontiguousarray(m.x0), np.ascontiguousarray(m.h)]
    ops_keep.extend(keep)
    v = bf.VolumeDesc()
    v.dim, v.N, v.K = m.dim, m.N, m.K
    v.r, v.w, v.Dr = (bf._dp(a) for a in (r, w, D))
    v.vmapM = m.vmapM.ctypes.data_as(bf.i32p)
    v.vmapP = m.vmapP.ctypes.data_as(bf.i32p)
    v.x0, v.h = bf._dp(keep[6]), bf._dp(keep[7])
    v.rho, v.lambda_, v.mu = bf._dp(rho), bf._dp(lam), bf._dp(mu)
    return v


def _create(v, g=None):
    opt = bf.Options()
    h = C.c_void_p()
    rc = bf.lib().bfam_gpu_domain_create(C.byref(v), C.byref(g) if g else None,
                                         C.byref(opt), C.byref(h))
    return rc, h


def test_rejects_corrupt_vmapP():
    m = bf.Mesh(3, 2, (2, 2, 2))
    keep = []
    v = _vol(m, keep)
    bad = m.vmapP.copy()
    bad[5] = bad[6]  # not a face of the element
    v.vmapP = bad.ctypes.data_as(bf.i32p)
    rc, _ = _create(v)
    assert rc == -1 and "vmapP" in bf.last_error()


def test_rejects_noncanonical_vmapM():
    m = bf.Mesh(2, 2, (3, 3))
    keep = []
    v = _vol(m, keep)
    bad = m.vmapM.copy()
    bad[0] += 1
    v.vmapM = bad.ctypes.data_as(bf.i32p)
    rc, _ = _create(v)
    assert rc == -1 and "vmapM" in bf.last_error()


def test_rejects_missing_glue():
    m = bf.Mesh(3, 2, (2, 2, 2), refine_prob=0.5, seed=1)
    assert m.Kg > 0
    keep = []
    v = _vol(m, keep)
    rc, _ = _create(v)  # hanging faces but no glue grid
    assert rc == -1 and "glue" in bf.last_error()


def test_rejects_broken_glue_involution():
    m = bf.Mesh(3, 2, (2, 2, 2), refine_prob=0.5, seed=1)
    keep = []
    v = _vol(m, keep)
    ops = bf.mortar_operators(2, 2)
    g = bf.GlueDesc()
    ep = m.EToEp.copy()
    ep[0], ep[1] = ep[1], ep[0]
    keep += [ep, ops]
    g.K = m.Kg
    g.EToEp = ep.ctypes.data_as(bf.i32p)
    for name in ("EToHp", "EToOp", "EToFm", "EToHm"):
        setattr(g, name, getattr(m, name).ctypes.data_as(bf.i8p))
    g.EToEm = m.EToEm.ctypes.data_as(bf.i32p)
    for s, k in enumerate((0, 3, 4)):
        g.interpolation[s] = bf._dp(ops[k]) if k else bf.dp()
    for s, k in enumerate((0, 1, 2)):
        g.projection[s] = bf._dp(ops[k]) if k else bf.dp()
    rc, _ = _create(v, g)
    assert rc == -1 and ("involution" in bf.last_error() or "EToHp" in bf.last_error())


def test_rejects_bad_material_and_order():
    m = bf.Mesh(2, 2, (2, 2))
    keep = []
    v = _vol(m, keep)
    mu0 = np.zeros(m.K)
    keep.append(mu0)
    v.mu = bf._dp(mu0)
    rc, _ = _create(v)
    assert rc == -1 and "mu" in bf.last_error()
    v2 = _vol(bf.Mesh(3, 9, (1, 1, 1)), keep)
    rc, _ = _create(v2)
    assert rc == -5


def test_batch_and_extras_reject_bad_arguments_without_a_device():
    L = bf.lib()
    h = C.c_void_p()
    assert L.bfam_gpu_batch_create(None, 0, 0, None, C.byref(h)) == bf.BFAM_GPU_EINVAL
    assert L.bfam_gpu_batch_create(None, 1, 0, None, None) == bf.BFAM_GPU_EINVAL
    assert L.bfam_gpu_batch_step(None, None, 1, 1) == bf.BFAM_GPU_EINVAL
    assert L.bfam_gpu_batch_set_tile(None, 0, 0, 0) == bf.BFAM_GPU_EINVAL
    assert L.bfam_gpu_batch_num_groups(None) == 0
    assert L.bfam_gpu_batch_free(None) == 0
    assert L.bfam_gpu_domain_set_source(None, None) == bf.BFAM_GPU_EINVAL
    assert L.bfam_gpu_domain_set_receivers(None, 1, None, 1) == bf.BFAM_GPU_EINVAL
    n = C.c_int()
    assert L.bfam_gpu_domain_get_seismograms(None, None, C.byref(n)) == bf.BFAM_GPU_EINVAL


def test_tile_table():
    # tile 0 is the single-domain kernel's shape (one element per CTA, one
    # thread per face node at least); the others may put several elements
    # in a CTA, down to one warp per element
    for dim, orders in ((2, range(1, 9)), (3, range(1, 8))):
        for N in orders:
            shapes = bf.tile_shapes(dim, N)
            epc = bf.tile_elements(dim, N)
            assert shapes and len(epc) == len(shapes), (dim, N)
            nfp = (N + 1) ** (dim - 1)
            assert shapes[0][0] >= 2 * dim * nfp and epc[0] == 1
            for (threads, minb), e in zip(shapes, epc):
                assert threads % 32 == 0 and minb >= 1 and e >= 1
                assert threads * e <= 1024
    assert bf.tile_elements(3, 3).count(1) == 3 and max(bf.tile_elements(3, 3)) == 4
    assert len(bf.tile_shapes(3, 5)) == 6 and len(bf.tile_shapes(3, 7)) == 2
    assert bf.lib().bfam_gpu_tile_count(3, 9) == 0
    a, b = C.c_int(), C.c_int()
    assert bf.lib().bfam_gpu_tile_shape(3, 5, 7, C.byref(a), C.byref(b)) == bf.BFAM_GPU_EINVAL
    assert bf.lib().bfam_gpu_tile_elements(3, 5, 7) == bf.BFAM_GPU_EINVAL


def test_autotune_cache_key_names_the_tile_table():
    """a cached tile index is only reused by a library with the same tile
    table for the order (the key lists every tile's shape)"""
    from bfam_b200 import autotune
    k5 = autotune._key("B200", 3, 5, 1)
    shapes = bf.tile_shapes(3, 5)
    assert k5.startswith("B200|dim3|N5|prec1|tiles:")
    assert k5.count("x") == 2 * len(shapes) and f"{shapes[0][0]}x{shapes[0][1]}x1" in k5
    assert autotune._key("B200", 3, 3, 1) != autotune._key("B200", 3, 5, 1)
