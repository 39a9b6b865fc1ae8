"""Brick mesher: bfam data-model invariants and geometric neighbours."""
from __future__ import annotations

import numpy as np
import pytest

import bfam_b200 as bf


def gmask(dim, Nq, f, pn):
    N = Nq - 1
    if dim == 2:
        return [pn * Nq, pn * Nq + N, pn, N * Nq + pn][f]
    a, b = pn % Nq, pn // Nq
    return [Nq * a + Nq * Nq * b, N + Nq * a + Nq * Nq * b, a + Nq * Nq * b,
            a + Nq * N + Nq * Nq * b, a + Nq * b, a + Nq * b + Nq * Nq * N][f]


def owner_map(m):
    D = [2 * m.nbase[0], 2 * m.nbase[1], 2 * m.nbase[2] if m.dim == 3 else 1]
    own = -np.ones(D[::-1], dtype=np.int64)  # [z][y][x]
    for e, (x, y, z, s) in enumerate(m.ecoord):
        if m.dim == 2:
            own[0, y:y + s, x:x + s] = e
        else:
            own[z:z + s, y:y + s, x:x + s] = e
    assert (own >= 0).all()
    return own, D


@pytest.mark.parametrize("dim,n,p,N", [(2, (4, 4), 0.0, 3), (2, (5, 3), 0.4, 2),
                                       (3, (4, 4, 4), 0.3, 2), (3, (3, 2, 5), 0.5, 1),
                                       (3, (2, 2, 2), 1.0, 2)])
def test_neighbours_are_geometric(dim, n, p, N):
    m = bf.Mesh(dim, N, n, refine_prob=p, seed=7)
    own, D = owner_map(m)
    NF = 2 * dim
    glue_faces = set(zip(m.EToEm.tolist(), m.EToFm.tolist()))
    for e in range(m.K):
        x = list(m.ecoord[e, :3])
        s = m.ecoord[e, 3]
        for f in range(NF):
            a, side = f // 2, f % 2
            pt = list(x)
            pt[a] = x[a] + s if side else x[a] - 1
            idx = [pt[i] % D[i] for i in range(3)] if dim == 3 else [pt[0] % D[0], pt[1] % D[1], 0]
            nb = own[idx[2], idx[1], idx[0]]
            if m.ecoord[nb, 3] == s:
                assert m.EToE[e, f] == nb and m.EToF[e, f] == (f ^ 1)
                assert (e, f) not in glue_faces
            else:
                assert m.EToE[e, f] == e and m.EToF[e, f] == f
                assert (e, f) in glue_faces


@pytest.mark.parametrize("dim", [2, 3])
def test_glue_receive_order_and_involution(dim):
    m = bf.Mesh(dim, 3, (4,) * dim, refine_prob=0.35, seed=3)
    assert m.Kg > 0
    keys = list(zip(m.EToEm.tolist(), m.EToFm.tolist(), m.EToHm.tolist()))
    assert keys == sorted(keys)
    g = np.arange(m.Kg)
    assert np.array_equal(m.EToEp[m.EToEp], g)
    assert np.array_equal(m.EToHp, m.EToHm[m.EToEp])
    assert (m.EToOp == 0).all()
    npc = 4 if dim == 3 else 2
    counts = np.bincount(m.EToHm, minlength=npc + 1)
    assert counts[0] == counts[1:].sum() and len(set(counts[1:])) == 1
    # partner of a hanging piece is the fine element on the other side
    for k in range(m.Kg):
        if m.EToHm[k] > 0:
            pe = m.EToEm[m.EToEp[k]]
            assert m.ecoord[pe, 3] * 2 == m.ecoord[m.EToEm[k], 3]
            assert m.EToFm[m.EToEp[k]] == (m.EToFm[k] ^ 1)


@pytest.mark.parametrize("dim", [2, 3])
def test_vmaps_follow_face_masks(dim):
    m = bf.Mesh(dim, 2, (3,) * dim, refine_prob=0.5, seed=11)
    Nq, Nfp, Np, NF = m.Nq, m.Nfp, m.Np, m.Nfaces
    vM = m.vmapM.reshape(m.K, NF, Nfp)
    vP = m.vmapP.reshape(m.K, NF, Nfp)
    for e in range(m.K):
        for f in range(NF):
            assert all(vM[e, f, q] == e * Np + gmask(dim, Nq, f, q) for q in range(Nfp))
            nb, nf = m.EToE[e, f], m.EToF[e, f]
            assert all(vP[e, f, q] == nb * Np + gmask(dim, Nq, nf, q) for q in range(Nfp))


def test_refinement_draw_is_seeded():
    a = bf.Mesh(3, 1, (8, 8, 8), refine_prob=0.3, seed=0)
    b = bf.Mesh(3, 1, (8, 8, 8), refine_prob=0.3, seed=0)
    c = bf.Mesh(3, 1, (8, 8, 8), refine_prob=0.3, seed=1)
    assert np.array_equal(a.ecoord, b.ecoord)
    assert not np.array_equal(a.ecoord, c.ecoord)
    assert a.K == 512 + 7 * a.num_refined


def test_mesh_rejects_bad_specs():
    with pytest.raises(ValueError):
        bf.Mesh(4, 3, (2, 2, 2))
    with pytest.raises(ValueError):
        bf.Mesh(3, 0, (2, 2, 2))
    with pytest.raises(ValueError):
        bf.Mesh(3, 3, (0, 2, 2))


def test_node_coordinates_cover_domain():
    m = bf.Mesh(3, 3, (2, 3, 4), L=(1.0, 2.0, 3.0), refine_prob=0.5, seed=2)
    r = bf.lgl_operators(3)[0]
    x, y, z = m.node_coordinates(r)
    assert np.isclose(x.min(), 0) and np.isclose(x.max(), 1)
    assert np.isclose(y.max(), 2) and np.isclose(z.max(), 3)
    # element volumes tile the domain
    assert np.isclose(np.prod(m.h, axis=1).sum(), 6.0)
