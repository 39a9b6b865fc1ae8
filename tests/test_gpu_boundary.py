"""Free-surface and absorbing boundary faces on the GPU, through the
bfam_gpu C-ABI (bfam_gpu_domain_create_with_boundary), against the oracle.

Bar: FP64 plain form to 1e-12 relative L2 per field (right-hand side, and
state after LSRK steps); the precision form to 1e-6 of the whole state."""
from __future__ import annotations

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from oracle import oracle as orc
from conftest import relerr
from test_boundary import _p_pulse

pytestmark = pytest.mark.gpu

TOL = 1e-12

CASES = [
    # dim, N, base cells, refine prob, seed, periodic, bc per side
    (2, 4, (6, 5), 0.4, 1, (False, True), 0),
    (2, 3, (4, 4), 0.5, 2, (False, False), (0, 1, 1, 0)),
    (3, 1, (3, 3, 3), 0.5, 3, (False, False, False), 1),
    (3, 3, (3, 2, 4), 0.4, 4, (False, True, False), (1, 0, 0, 0, 0, 1)),
    (3, 5, (3, 3, 3), 0.3, 6, (True, False, True), 0),
    (3, 5, (2, 2, 2), 1.0, 9, (False, False, False), (0, 1, 0, 1, 0, 1)),
    (3, 7, (2, 3, 2), 0.5, 8, (False, False, False), 0),
    (3, 4, (1, 1, 1), 0.0, 0, (False, False, False), 1),  # one element, all sides
]


def _setup(dim, N, n, p, seed, periodic, bc):
    m = bf.Mesh(dim, N, n, refine_prob=p, seed=seed, periodic=periodic)
    rho, lam, mu = bf.material_random(m.K, seed + 10)
    return m, rho, lam, mu


def _id(c):
    return f"{c[0]}d-N{c[1]}-{'x'.join(map(str, c[2]))}-p{c[3]}-bc{c[6]}"


@pytest.mark.parametrize("case", CASES, ids=_id)
@pytest.mark.parametrize("flux", [0, 1], ids=["upwind", "central"])
def test_rhs_parity_with_boundaries(case, flux):
    m, rho, lam, mu = _setup(*case)
    assert m.Kb > 0
    rng = np.random.default_rng(case[4])
    q = rng.standard_normal((m.nfields, m.K * m.Np))
    dom = bf.GpuDomain(m, rho, lam, mu, flux=flux, bc=case[6])
    dom.set_fields(q)
    got = dom.rhs()
    ref = orc.Oracle.from_mesh(m, rho, lam, mu, flux, bc=case[6]).rhs(q)
    assert relerr(got, ref).max() < TOL


@pytest.mark.parametrize("case", [CASES[1], CASES[3], CASES[4], CASES[6]], ids=_id)
def test_lsrk_parity_with_boundaries(case):
    m, rho, lam, mu = _setup(*case)
    r = bf.lgl_operators(m.N)[0]
    q0 = m.gaussian_pulse(r, (0.8, 0.3, 0.6), 0.2)
    dt = configs.stable_dt(m, rho, lam, mu, 0.5)
    dom = bf.GpuDomain(m, rho, lam, mu, bc=case[6])
    dom.set_fields(q0)
    ts = bf.LSRK(dom)
    ts.step(dt, 20, use_graph=True)
    got = dom.get_fields()
    o = orc.Oracle.from_mesh(m, rho, lam, mu, bc=case[6])
    ref = o.lsrk(q0, dt, 20)
    assert relerr(got, ref).max() < TOL
    assert abs(dom.energy() - o.energy(ref)) < 1e-12 * o.energy(ref)


@pytest.mark.parametrize("bc", [bf.BC_FREE_SURFACE, bf.BC_ABSORBING])
def test_p_pulse_reflects_or_leaves_on_gpu(bc):
    """Normal-incidence P pulse at x = 1: the free surface reflects it as
    v_x = f(2 - x - ct), sxx = rho c v_x, syy = (lam / c) v_x; the absorbing
    side lets it leave"""
    N, T = 6, 0.4
    m = bf.Mesh(2, N, (20, 2), periodic=(False, True))
    r = bf.lgl_operators(N)[0]
    q0, c = _p_pulse(m, r, 0.5, 0.06, 1.0, 2.0, 1.0)
    dt0 = configs.stable_dt(m, 1.0, 2.0, 1.0, 0.4)
    steps = int(np.ceil(T / dt0))
    dom = bf.GpuDomain(m, 1.0, 2.0, 1.0, bc=bc)
    dom.set_fields(q0)
    E0 = dom.energy()
    bf.LSRK(dom).step(T / steps, steps, use_graph=True)
    q = dom.get_fields()
    if bc == bf.BC_ABSORBING:
        assert dom.energy() < 1e-12 * E0
        return
    x, _, _ = m.node_coordinates(r)
    g = np.exp(-(((2 - x - c * T) - 0.5) / 0.06) ** 2)
    qe = np.zeros_like(q)
    qe[0], qe[2], qe[3] = g, c * g, (2.0 / c) * g
    assert np.sqrt(((q - qe) ** 2).sum() / (qe ** 2).sum()) < 1e-4
    assert dom.energy() > 0.9999 * E0


def test_precision_form_with_boundaries():
    m, rho, lam, mu = _setup(*CASES[4])
    r = bf.lgl_operators(m.N)[0]
    q0 = m.gaussian_pulse(r, (0.5, 0.9, 0.5), 0.2)
    dt = configs.stable_dt(m, rho, lam, mu, 0.5)
    dom = bf.GpuDomain(m, rho, lam, mu, precision=bf.PRECISION_FP32, bc=CASES[4][6])
    dom.set_fields(q0)
    bf.LSRK(dom).step(dt, 20)
    got = dom.get_fields()
    ref = orc.Oracle.from_mesh(m, rho, lam, mu, bc=CASES[4][6]).lsrk(q0, dt, 20)
    err = np.sqrt(((got - ref) ** 2).sum() / (ref ** 2).sum())
    assert err < 1e-6, err


def test_batch_with_boundary_domains_equals_alone():
    probs = [CASES[3], CASES[4], CASES[0]]
    alone, doms = [], []
    for c in probs:
        m, rho, lam, mu = _setup(*c)
        r = bf.lgl_operators(m.N)[0]
        q0 = m.gaussian_pulse(r, (0.2, 0.5, 0.5), 0.2)
        dt = configs.stable_dt(m, rho, lam, mu, 0.5)
        d = bf.GpuDomain(m, rho, lam, mu, bc=c[6])
        d.set_fields(q0)
        bf.LSRK(d).step(dt, 10)
        alone.append(d.get_fields())
        d.free()
        d = bf.GpuDomain(m, rho, lam, mu, bc=c[6])
        d.set_fields(q0)
        doms.append((d, dt))
    b = bf.Batch([d for d, _ in doms])
    b.step([dt for _, dt in doms], 10)
    b.sync()
    for (d, _), a in zip(doms, alone):
        assert np.array_equal(d.get_fields(), a)
    b.free()
