"""Boundary faces of non-periodic bricks (the role of bfam's boundary glue
grids, src/bfam.c:7851-7899): the mesher's boundary list, the C-ABI's
checks of it, and the oracle's free-surface and absorbing conditions
against known answers."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from oracle import oracle as orc
from test_mesh import owner_map


@pytest.mark.parametrize("dim,n,p,periodic", [
    (2, (5, 3), 0.4, (False, True)),
    (2, (4, 4), 0.0, (False, False)),
    (3, (3, 2, 4), 0.5, (False, True, False)),
    (3, (2, 2, 2), 1.0, (False, False, False)),
    (3, (4, 3, 3), 0.3, (True, False, True)),
])
def test_boundary_faces_are_the_brick_sides(dim, n, p, periodic):
    m = bf.Mesh(dim, 2, n, refine_prob=p, seed=5, periodic=periodic)
    own, D = owner_map(m)
    NF = 2 * dim
    bset = set(zip(m.EToEb.tolist(), m.EToFb.tolist()))
    assert len(bset) == m.Kb
    glue = set(zip(m.EToEm.tolist(), m.EToFm.tolist()))
    area = np.zeros(NF)
    for e in range(m.K):
        x = list(m.ecoord[e, :3])
        s = m.ecoord[e, 3]
        for f in range(NF):
            a, side = f // 2, f % 2
            out = x[a] + s if side else x[a] - 1
            on_side = not periodic[a] and (out < 0 or out >= D[a])
            assert ((e, f) in bset) == on_side
            if on_side:
                assert m.EToE[e, f] == e and m.EToF[e, f] == f
                assert (e, f) not in glue
                area[f] += s ** (dim - 1)
    # every side of a non-periodic axis is covered exactly once
    for f in range(NF):
        a = f // 2
        full = np.prod([D[b] for b in range(dim) if b != a])
        assert area[f] == (0 if periodic[a] else full)


def _vol(m, keep):
    r, w, wi, D = bf.lgl_operators(m.N)
    rho, lam, mu = np.ones(m.K), np.full(m.K, 2.0), np.ones(m.K)
    x0, h = np.ascontiguousarray(m.x0), np.ascontiguousarray(m.h)
    keep += [r, w, D, rho, lam, mu, x0, h]
    v = bf.VolumeDesc()
    v.dim, v.N, v.K = m.dim, m.N, m.K
    v.r, v.w, v.Dr = (bf._dp(a) for a in (r, w, D))
    v.vmapM = m.vmapM.ctypes.data_as(bf.i32p)
    v.vmapP = m.vmapP.ctypes.data_as(bf.i32p)
    v.x0, v.h = bf._dp(x0), bf._dp(h)
    v.rho, v.lambda_, v.mu = bf._dp(rho), bf._dp(lam), bf._dp(mu)
    return v


def _create(m, E, F, T):
    keep = []
    v = _vol(m, keep)
    E, F, T = (np.ascontiguousarray(a, dtype=t) for a, t in
               ((E, np.int32), (F, np.int8), (T, np.int8)))
    b = bf.BoundaryDesc()
    b.K = len(E)
    b.EToE = E.ctypes.data_as(bf.i32p)
    b.EToF = F.ctypes.data_as(bf.i8p)
    b.type = T.ctypes.data_as(bf.i8p)
    g = bf.GlueDesc()
    opt = bf.Options()
    h = C.c_void_p()
    rc = bf.lib().bfam_gpu_domain_create_with_boundary(
        C.byref(v), C.byref(g), C.byref(b), C.byref(opt), C.byref(h))
    return rc


def test_abi_rejects_bad_boundary_lists():
    m = bf.Mesh(3, 2, (2, 2, 2), periodic=(False, True, True))
    assert m.Kg == 0 and m.Kb == 8
    E, F = m.EToEb, m.EToFb
    T = np.zeros(m.Kb, dtype=np.int8)
    # the boundary list missing: self-mapped faces with nothing behind them
    keep = []
    v = _vol(m, keep)
    h = C.c_void_p()
    rc = bf.lib().bfam_gpu_domain_create(C.byref(v), None, C.byref(bf.Options()),
                                         C.byref(h))
    assert rc == -1 and "boundary entry" in bf.last_error()
    # one face left out
    assert _create(m, E[1:], F[1:], T[1:]) == -1
    assert "boundary entry" in bf.last_error()
    # unknown condition
    T2 = T.copy()
    T2[3] = 7
    assert _create(m, E, F, T2) == -1 and "unknown type" in bf.last_error()
    # the same face twice
    E2, F2 = np.append(E, E[0]), np.append(F, F[0])
    assert _create(m, E2, F2, np.zeros(m.Kb + 1)) == -1
    assert "second boundary entry" in bf.last_error()
    # an interior face (it has a neighbour)
    F3 = F.copy()
    F3[0] = 2
    assert _create(m, E, F3, T) == -1 and "has a neighbour" in bf.last_error()
    # face number out of range
    F4 = F.copy()
    F4[0] = 6
    assert _create(m, E, F4, T) == -1 and "bad (E, F)" in bf.last_error()


# ---------------------------------------------------------------- oracle

def _p_pulse(m, r, x0, w, rho, lam, mu):
    """right-going P pulse v_x = exp(-((x - x0) / w)^2) in 2D, with its
    stresses sxx = -rho c v_x, syy = -(lam / c) v_x"""
    c = math.sqrt((lam + 2 * mu) / rho)
    x, _, _ = m.node_coordinates(r)
    f = np.exp(-(((x - x0) / w) ** 2))
    q = np.zeros((5, m.K * m.Np))
    q[0] = f
    q[2] = -rho * c * f
    q[3] = -(lam / c) * f
    return q, c


def _run(o, q, T, m, cfl=0.4):
    dt0 = configs.stable_dt(m, 1.0, 2.0, 1.0, cfl)
    steps = int(math.ceil(T / dt0))
    return o.lsrk(q, T / steps, steps)


def test_free_surface_reflects_a_p_pulse_with_traction_zero():
    """Normal-incidence P pulse on the free surface x = 1: the reflected
    pulse is v_x = f(2 - x - ct), sxx = +rho c v_x, syy = +(lam / c) v_x."""
    N = 6
    m = bf.Mesh(2, N, (20, 2), periodic=(False, True))
    r = bf.lgl_operators(N)[0]
    q0, c = _p_pulse(m, r, 0.5, 0.06, 1.0, 2.0, 1.0)
    o = orc.Oracle.from_mesh(m, 1.0, 2.0, 1.0, bc=bf.BC_FREE_SURFACE)
    T = 0.4
    q = _run(o, q0, T, m)
    x, _, _ = m.node_coordinates(r)
    g = np.exp(-(((2 - x - c * T) - 0.5) / 0.06) ** 2)
    qe = np.zeros_like(q)
    qe[0] = g
    qe[2] = c * g
    qe[3] = (2.0 / c) * g
    err = np.sqrt(((q - qe) ** 2).sum() / (qe ** 2).sum())
    assert err < 1e-4, err
    # the reflection lost (almost) no energy
    assert o.energy(q) > 0.9999 * o.energy(q0)


def test_absorbing_boundary_lets_a_p_pulse_leave():
    N = 6
    m = bf.Mesh(2, N, (20, 2), periodic=(False, True))
    r = bf.lgl_operators(N)[0]
    q0, c = _p_pulse(m, r, 0.5, 0.06, 1.0, 2.0, 1.0)
    o = orc.Oracle.from_mesh(m, 1.0, 2.0, 1.0, bc=bf.BC_ABSORBING)
    q = _run(o, q0, 0.4, m)
    assert o.energy(q) < 1e-12 * o.energy(q0)


def test_free_surface_keeps_a_rigid_motion_at_rest():
    """constant velocity with zero stress satisfies the free-surface
    condition: the right-hand side vanishes (on hanging meshes too)"""
    m = bf.Mesh(3, 3, (3, 2, 3), refine_prob=0.5, seed=1, periodic=(False, False, False))
    rho, lam, mu = bf.material_random(m.K, 1)
    q = np.zeros((9, m.K * m.Np))
    q[0], q[1], q[2] = 0.3, -1.2, 2.0
    rhs = orc.Oracle.from_mesh(m, rho, lam, mu, bc=bf.BC_FREE_SURFACE).rhs(q)
    assert np.abs(rhs).max() < 1e-10
    # the absorbing condition drags the same state at the sides
    rhs = orc.Oracle.from_mesh(m, rho, lam, mu, bc=bf.BC_ABSORBING).rhs(q)
    assert np.abs(rhs).max() > 1e-2


@pytest.mark.parametrize("bc", [bf.BC_FREE_SURFACE, bf.BC_ABSORBING,
                                (0, 1, 1, 0, 0, 1)])
def test_energy_decays_with_boundaries_and_mortars(bc):
    m = bf.Mesh(3, 3, (3, 3, 3), refine_prob=0.4, seed=2, periodic=(False, True, False))
    r = bf.lgl_operators(3)[0]
    rho, lam, mu = bf.material_random(m.K, 3)
    q = m.gaussian_pulse(r, (0.8, 0.5, 0.2), 0.2)
    o = orc.Oracle.from_mesh(m, rho, lam, mu, bc=bc)
    dt = configs.stable_dt(m, rho, lam, mu, 0.5)
    E = [o.energy(q)]
    for _ in range(6):
        q = o.lsrk(q, dt, 4)
        E.append(o.energy(q))
    assert np.all(np.diff(E) < 0)
