"""The oracle against known answers: analytic plane waves (order N+1),
the discrete energy identity, and symmetry/conservation properties."""
from __future__ import annotations

import math

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from oracle import oracle as orc
from conftest import relerr


def _pw_error(dim, n, N, T, refine=0.0, cfl=0.25, k=None):
    m = bf.Mesh(dim, N, (n,) * dim, refine_prob=refine, seed=0)
    r = bf.lgl_operators(N)[0]
    k = k or ((2 * math.pi, 2 * math.pi) if dim == 2 else (2 * math.pi, 0.0, 0.0))
    o = orc.Oracle.from_mesh(m, 1.0, 2.0, 1.0)
    q0 = m.plane_wave(r, k, 1.0, 1.0, 2.0, 1.0, 0.0)
    dt0 = configs.stable_dt(m, 1.0, 2.0, 1.0, cfl)
    steps = int(math.ceil(T / dt0))
    q = o.lsrk(q0, T / steps, steps)
    qe = m.plane_wave(r, k, 1.0, 1.0, 2.0, 1.0, T)
    return np.sqrt(((q - qe) ** 2).sum() / (qe ** 2).sum())


@pytest.mark.parametrize("N", [2, 3, 4])
def test_2d_plane_wave_converges_at_order_N_plus_1(N):
    e1 = _pw_error(2, 4, N, 0.1)
    e2 = _pw_error(2, 8, N, 0.1)
    rate = math.log2(e1 / e2)
    assert rate > N + 1 - 0.4, (e1, e2, rate)


def _pw_error_halfrefined(n, N, T, k):
    """Base cells with x < 1/2 refined: nested meshes whose hanging faces
    (at x = 0 and x = 1/2) cross the wave."""
    flags = np.zeros((n, n, n), dtype=np.uint8)
    flags[:, :, : n // 2] = 1  # [z][y][x]
    m = bf.Mesh(3, N, (n, n, n), refine_flags=flags.reshape(-1))
    assert m.Kg > 0
    r = bf.lgl_operators(N)[0]
    o = orc.Oracle.from_mesh(m, 1.0, 2.0, 1.0)
    q0 = m.plane_wave(r, k, 1.0, 1.0, 2.0, 1.0, 0.0)
    dt0 = configs.stable_dt(m, 1.0, 2.0, 1.0, 0.25)
    steps = int(math.ceil(T / dt0))
    q = o.lsrk(q0, T / steps, steps)
    qe = m.plane_wave(r, k, 1.0, 1.0, 2.0, 1.0, T)
    return np.sqrt(((q - qe) ** 2).sum() / (qe ** 2).sum())


def test_3d_mortar_plane_wave_converges():
    """Oblique wave through nested meshes with mortars: rate near N+1."""
    N, k = 3, (2 * math.pi, 0.0, 0.0)
    e1 = _pw_error_halfrefined(2, N, 0.05, k)
    e2 = _pw_error_halfrefined(4, N, 0.05, k)
    assert math.log2(e1 / e2) > N + 1 - 0.5, (e1, e2)


def test_cfg0_matches_analytic():
    p = configs.cfg0()
    o = orc.Oracle.from_mesh(p.mesh, p.rho, p.lam, p.mu)
    q = o.lsrk(p.q0, p.dt, p.nsteps)
    r = bf.lgl_operators(p.mesh.N)[0]
    qe = p.mesh.plane_wave(r, p.meta["k"], 1.0, 1.0, 2.0, 1.0, p.dt * p.nsteps)
    assert relerr(q, qe).max() < 1e-5


def test_energy_upwind_decays_with_mortars():
    m = bf.Mesh(3, 3, (4, 4, 4), refine_prob=0.3, seed=0)
    r = bf.lgl_operators(3)[0]
    rho, lam, mu = bf.material_random(m.K, 0)
    q = m.gaussian_pulse(r, (0.5, 0.5, 0.5), 0.15)
    o = orc.Oracle.from_mesh(m, rho, lam, mu, flux=0)
    dt = configs.stable_dt(m, rho, lam, mu, 0.5)
    E = [o.energy(q)]
    for _ in range(8):
        q = o.lsrk(q, dt, 4)
        E.append(o.energy(q))
    assert np.all(np.diff(E) < 0)


def test_energy_central_conserved_conforming():
    m = bf.Mesh(3, 3, (3, 3, 3))
    r = bf.lgl_operators(3)[0]
    rng = np.random.default_rng(0)
    rho, lam, mu = bf.material_random(m.K, 5)
    q = m.gaussian_pulse(r, (0.4, 0.5, 0.6), 0.2)
    o = orc.Oracle.from_mesh(m, rho, lam, mu, flux=1)
    E0 = o.energy(q)
    dt = configs.stable_dt(m, rho, lam, mu, 0.25)
    q = o.lsrk(q, dt, 20)
    # RK4 damps skew-symmetric dynamics by O(dt^4) only
    assert abs(o.energy(q) - E0) / E0 < 1e-6


def test_rhs_of_constant_state_vanishes():
    """Constant fields are in the kernel of the operator (free-stream)."""
    m = bf.Mesh(3, 3, (3, 3, 3), refine_prob=0.5, seed=1)
    rho, lam, mu = bf.material_random(m.K, 1)
    q = np.ones((9, m.K * m.Np))
    rhs = orc.Oracle.from_mesh(m, 1.0, 2.0, 1.0).rhs(q)
    assert np.abs(rhs).max() < 1e-10


def test_rhs_linear():
    m = bf.Mesh(2, 3, (3, 4), refine_prob=0.5, seed=4)
    rho, lam, mu = bf.material_random(m.K, 4)
    o = orc.Oracle.from_mesh(m, rho, lam, mu)
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal((2, 5, m.K * m.Np))
    lhs = o.rhs(2.0 * a - 3.0 * b)
    rhs = 2.0 * o.rhs(a) - 3.0 * o.rhs(b)
    assert np.abs(lhs - rhs).max() < 1e-9 * np.abs(rhs).max()
