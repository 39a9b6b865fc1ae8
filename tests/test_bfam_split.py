"""The drop-in's input format pinned against bfam itself (CPU).

The reference's whole src/bfam.c and its vendored p4est-1.1 are compiled from
source into oracle/_ref/ (oracle/build_ref.sh); oracle/bfam_ref.py runs bfam's
own front end (p4est brick, seeded refinement, 2:1 balance,
bfam_domain_pxest_split_dgx_subdomains, src/bfam.c:7565-8054) and returns the
arrays bfam holds.  Checked here:
  * the repository's brick mesher emits exactly bfam's arrays (vmapM, vmapP,
    the glue grid's EToEm/EToFm/EToHm/EToEp/EToHp/EToOp in bfam's receive
    order, the boundary glue grid's faces), including the hanging-piece
    numbering that bfam derives with BFAM_PXEST_BOHTONH (src/bfam.c:3719-3728,
    4721, 4786);
  * bfam's LGL and glue operators equal the ones the product computes;
  * the oracle runs on bfam's multi-level forests (several refinement
    levels, hanging faces between every pair of adjacent levels) and gives
    known answers there: zero right-hand side for a constant state, and
    decaying discrete energy under the upwind flux.
"""
from __future__ import annotations

import numpy as np
import pytest

import bfam_b200 as bf
from oracle import bfam_ref as br
from oracle import oracle as orc

pytestmark = pytest.mark.skipif(not (br.available(2) and br.available(3)),
                                reason="oracle/_ref/libbfam_ref{2,3}d.so not built")

MESHER_CASES = [
    # dim, base cells, N, seed, refine prob, periodic
    (2, (6, 5), 1, 0, 0.3, (1, 1)),
    (2, (5, 3), 4, 3, 0.4, (1, 0)),
    (2, (4, 4), 3, 7, 1.0, (0, 0)),
    (3, (4, 4, 4), 3, 0, 0.3, (1, 1, 1)),
    (3, (3, 5, 2), 2, 3, 0.4, (0, 1, 0)),
    (3, (4, 4, 4), 5, 1, 0.5, (0, 0, 0)),
    (3, (2, 3, 2), 7, 8, 0.5, (1, 1, 1)),
    (3, (1, 1, 1), 3, 0, 0.0, (1, 1, 1)),
]

GLUE = ("EToEm", "EToFm", "EToHm", "EToEp", "EToHp", "EToOp")


@pytest.mark.parametrize("case", MESHER_CASES,
                         ids=lambda c: f"{c[0]}d-{c[1]}-N{c[2]}-s{c[3]}-p{c[4]}-per{c[5]}")
def test_mesher_emits_bfams_split(case):
    dim, n, N, seed, prob, per = case
    ref = br.BfamMesh(dim, n, N, seed=seed, levels=1, prob=prob, periodic=per)
    m = bf.Mesh(dim, N, n, refine_prob=prob, seed=seed,
                periodic=tuple(bool(p) for p in per))
    assert (m.K, m.Kg, m.Kb) == (ref.K, ref.Kg, ref.Kb)
    assert ref.num_local_glue == (1 if ref.Kg else 0)
    assert np.array_equal(m.vmapM, ref.vmapM)
    assert np.array_equal(m.vmapP, ref.vmapP)
    for name in GLUE:
        assert np.array_equal(np.asarray(getattr(m, name)), getattr(ref, name)), name
    # boundary glue grid: same faces in the same order
    assert np.array_equal(m.EToEb, ref.EToEb) and np.array_equal(m.EToFb, ref.EToFb)
    # element boxes (bfam's quadrants in its brick) and finest-cell boxes
    assert np.allclose(m.x0[:, :dim], ref.x0[:, :dim], rtol=0, atol=1e-15)
    assert np.array_equal(m.h[:, :dim], ref.h[:, :dim])
    # (the mesher counts in half base cells; bfam's finest level may be 0)
    assert np.array_equal(np.asarray(m.ecoord).reshape(-1, 4),
                          ref.ecoord << (1 - ref.max_level))


def test_hanging_piece_numbering_is_bfams():
    """Piece h of a coarse face is 1 + a + 2b, a (b) the half along the
    face's first (second) tangential axis: bfam's numbering after its
    BOHTONH remap at orientation 0, read off bfam's own glue grid (a bounded
    brick, so that no face wraps around)."""
    tang = {0: (1, 2), 1: (0, 2), 2: (0, 1)}
    for dim, n in ((2, (5, 4)), (3, (4, 4, 4))):
        ref = br.BfamMesh(dim, n, 2, seed=0, levels=2, prob=0.3,
                          periodic=(0, 0, 0))
        checked = 0
        for g in range(ref.Kg):
            h = int(ref.EToHm[g])
            if h == 0:
                continue
            e, f = int(ref.EToEm[g]), int(ref.EToFm[g])
            fine = int(ref.EToEm[ref.EToEp[g]])
            rel = np.rint((ref.x0[fine, :dim] - ref.x0[e, :dim]) / ref.h[fine, :dim]).astype(int)
            t0, t1 = tang[f // 2] if dim == 3 else ((1, None) if f < 2 else (0, None))
            a = rel[t0]
            b = rel[t1] if t1 is not None else 0
            assert a in (0, 1) and b in (0, 1)
            assert h == 1 + a + 2 * b
            checked += 1
        assert checked > 0


def test_operators_equal_products():
    for N in (1, 3, 5, 7):
        ref = br.BfamMesh(3, (2, 2, 2), N, seed=1, levels=1, prob=0.5)
        r, w, _, Dr = bf.lgl_operators(N)
        assert np.array_equal(ref.r, r) and np.array_equal(ref.w, w)
        assert np.array_equal(ref.Dr, Dr)
        ops = bf.mortar_operators(N, N)  # same, cfb, cft, r2b, r2t
        assert ref.interp[0] is None and ref.proj[0] is None
        assert np.array_equal(ref.interp[1], ops[3]) and np.array_equal(ref.interp[2], ops[4])
        assert np.array_equal(ref.proj[1], ops[1]) and np.array_equal(ref.proj[2], ops[2])


MULTI = [
    # dim, base cells, N, seed, levels, prob
    (2, (4, 4), 3, 1, 3, 0.35),
    (3, (3, 3, 3), 2, 1, 2, 0.35),
    (3, (3, 3, 3), 2, 2, 3, 0.3),
]


@pytest.mark.parametrize("case", MULTI, ids=lambda c: f"{c[0]}d-{c[1]}-N{c[2]}-L{c[4]}")
def test_multilevel_forest(case):
    dim, n, N, seed, levels, prob = case
    ref = br.BfamMesh(dim, n, N, seed=seed, levels=levels, prob=prob)
    assert ref.max_level == levels
    assert len(np.unique(ref.level)) >= 2
    # glue grid: receive order, EToEp an involution, pieces pair with whole
    # faces, every face aligned (bricks have orientation 0)
    g = np.arange(ref.Kg)
    assert np.array_equal(ref.EToEp[ref.EToEp], g)
    assert np.array_equal(ref.EToHp, ref.EToHm[ref.EToEp])
    assert not np.any((ref.EToHm > 0) & (ref.EToHp > 0))
    assert not np.any(ref.EToOp)
    key = (ref.EToEm.astype(np.int64) * 8 + ref.EToFm) * 8 + ref.EToHm
    assert np.all(np.diff(key) > 0)
    # 2:1 across hanging faces; an element is fine on at most dim faces
    fine = ref.EToEm[ref.EToEp[ref.EToHm > 0]]
    coarse = ref.EToEm[ref.EToHm > 0]
    assert np.all(ref.level[fine] == ref.level[coarse] + 1)
    fine_faces = ref.EToEm[(ref.EToHm == 0) & (ref.EToHp > 0)]
    assert np.bincount(fine_faces, minlength=ref.K).max() <= dim
    # elements both fine (on one face) and coarse (on another) exist
    both = np.intersect1d(fine_faces, coarse)
    assert levels < 3 or both.size > 0

    # the oracle on this forest: constant state -> zero rhs; energy decays
    rho, lam, mu = bf.material_random(ref.K, seed + 20)
    o = orc.Oracle(dim, N, ref.ecoord, ref.nbase, ref.L, rho, lam, mu, 0, fine=ref.fine)
    const = np.ones((ref.nfields, ref.K * ref.Np)) * np.arange(1, ref.nfields + 1)[:, None]
    assert np.abs(o.rhs(const)).max() < 1e-10
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((ref.nfields, ref.K * ref.Np))
    from bfam_b200 import configs
    dt = configs.stable_dt(ref, rho, lam, mu, 0.3)
    e0 = o.energy(q)
    q1 = o.lsrk(q, dt, 3)
    assert o.energy(q1) < e0
