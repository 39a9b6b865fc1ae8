"""Glue between subdomains of different orders (p-nonconforming faces,
bfam's glue grid between two volume subdomains, src/bfam.c:7340-7414 with
the operators of 5471-5514 and 5607-5691).

CPU: the oracle's glue operators pinned to the reference's, the oracle's
glued subdomains against the unsplit brick (equal orders) and an analytic
plane wave (different orders).  GPU: two domains stepped in one batch with
their glue against the oracle (FP64 1e-12 per field; precision form 1e-6),
and the C-ABI's checks."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from oracle import oracle as orc
from conftest import relerr

GOLD = np.load(Path(__file__).parent / "golden" / "reference_ops.npz")


@pytest.mark.parametrize("pair", [(3, 5), (5, 7)])
def test_oracle_glue_operators_pinned(pair):
    """I = glue_m->interpolation[0] (order N to Ng), P = projection[0] back"""
    N, Ng = pair
    I, P = orc.glue_ops(N, Ng)
    n, m = N + 1, Ng + 1
    gI = GOLD[f"prj_{N}_to_{Ng}"][0].reshape(n, m).T   # column-major m x n
    gP = GOLD[f"prj_{Ng}_to_{N}"][0].reshape(m, n).T   # column-major n x m
    assert np.abs(I - gI).max() < 1e-14
    assert np.abs(P - gP).max() < 1e-13
    assert np.abs(P @ I - np.eye(n)).max() < 1e-13


def split_brick(dim, Na, Nb, n, seed=0, refine=0.0, nx=(2, 2)):
    """Two bricks of orders Na, Nb sharing their y/z extent, x in [0, 1/2)
    and [1/2, 1), glued along x into one periodic domain; base cells next
    to the glued sides are not refined (same-size glued faces)."""
    rng = np.random.default_rng(seed)
    meshes = []
    for N, nxi in zip((Na, Nb), nx):
        cells = (nxi,) + (n,) * (dim - 1)
        flags = (rng.random(cells[::-1]) < refine).astype(np.uint8)
        flags[..., 0] = 0
        flags[..., -1] = 0
        L = (0.5,) + (1.0,) * (dim - 1)
        meshes.append(bf.Mesh(dim, N, cells, L=L, refine_flags=flags.reshape(-1),
                              periodic=(False,) + (True,) * (dim - 1)))
    ma, mb = meshes
    ea, eb = bf.glued_x_pairs(ma, mb)
    pairs = np.stack([ma.EToEb[ea], ma.EToFb[ea], mb.EToEb[eb], mb.EToFb[eb]], axis=1)
    return ma, mb, ea, eb, pairs


def _glued_bc(m):
    return (bf.BC_GLUED, bf.BC_GLUED) + (bf.BC_FREE_SURFACE,) * (2 * m.dim - 2)


def _plane_wave(m, x_offset, t):
    """P wave k = (2 pi, 0, 0) in rho=1, lambda=2, mu=1 (cp = 2) at global
    x = local x + x_offset: the same wave at time t - x_offset / cp"""
    r = bf.lgl_operators(m.N)[0]
    k = (2 * math.pi,) + (0.0,) * (m.dim - 1)
    return m.plane_wave(r, k, 1.0, 1.0, 2.0, 1.0, t - x_offset / 2.0)


def test_equal_orders_glued_halves_equal_the_whole_brick():
    N, n = 3, 3
    ma, mb, ea, eb, pairs = split_brick(3, N, N, n, nx=(3, 3))
    whole = bf.Mesh(3, N, (6, n, n), L=(1.0, 1.0, 1.0))
    rng = np.random.default_rng(1)
    qa = rng.standard_normal((9, ma.K * ma.Np))
    qb = rng.standard_normal((9, mb.K * mb.Np))
    po = orc.PGlueOracle(orc.Oracle.from_mesh(ma, 1.0, 2.0, 1.0),
                         orc.Oracle.from_mesh(mb, 1.0, 2.0, 1.0), pairs)
    ra, rb = po.rhs(qa, qb)
    # the same fields on the whole brick: element (x, y, z) of a half is
    # element (x + 3 * half, y, z) of the whole
    def index(m, xoff):
        key = {tuple(c): e for e, c in enumerate(whole.ecoord[:, :3].tolist())}
        return np.array([key[(c[0] + xoff, c[1], c[2])] for c in m.ecoord[:, :3].tolist()])
    ia, ib = index(ma, 0), index(mb, 6)
    q = np.zeros((9, whole.K, whole.Np))
    q[:, ia] = qa.reshape(9, ma.K, ma.Np)
    q[:, ib] = qb.reshape(9, mb.K, mb.Np)
    r = orc.Oracle.from_mesh(whole, 1.0, 2.0, 1.0).rhs(q.reshape(9, -1)).reshape(9, whole.K, -1)
    assert relerr(ra, r[:, ia].reshape(9, -1)).max() < 1e-13
    assert relerr(rb, r[:, ib].reshape(9, -1)).max() < 1e-13


def _pw_error(Na, Nb, n, T=0.05):
    ma, mb, ea, eb, pairs = split_brick(3, Na, Nb, n, nx=(n // 2, n // 2))
    po = orc.PGlueOracle(orc.Oracle.from_mesh(ma, 1.0, 2.0, 1.0),
                         orc.Oracle.from_mesh(mb, 1.0, 2.0, 1.0), pairs)
    dt0 = min(configs.stable_dt(m, 1.0, 2.0, 1.0, 0.25) for m in (ma, mb))
    steps = int(math.ceil(T / dt0))
    qa, qb = po.lsrk(_plane_wave(ma, 0.0, 0.0), _plane_wave(mb, 0.5, 0.0), T / steps, steps)
    ea_ = _plane_wave(ma, 0.0, T)
    eb_ = _plane_wave(mb, 0.5, T)
    num = ((qa - ea_) ** 2).sum() + ((qb - eb_) ** 2).sum()
    den = (ea_ ** 2).sum() + (eb_ ** 2).sum()
    return math.sqrt(num / den)


def test_plane_wave_through_glue_of_orders_3_and_5_converges():
    """the wave crosses both glued sides; the error falls at the lower
    order's rate"""
    e1 = _pw_error(3, 5, 2)
    e2 = _pw_error(3, 5, 4)
    rate = math.log2(e1 / e2)
    assert rate > 3.5, (e1, e2, rate)
    # half the domain at order 5 beats order 3 everywhere
    assert e2 < 0.7 * _pw_error(3, 3, 4)


def test_energy_decays_across_glue_of_orders():
    ma, mb, ea, eb, pairs = split_brick(3, 2, 4, 3, refine=0.5, seed=3, nx=(3, 3))
    rho_a, lam_a, mu_a = bf.material_random(ma.K, 1)
    rho_b, lam_b, mu_b = bf.material_random(mb.K, 2)
    oa = orc.Oracle.from_mesh(ma, rho_a, lam_a, mu_a)
    ob = orc.Oracle.from_mesh(mb, rho_b, lam_b, mu_b)
    po = orc.PGlueOracle(oa, ob, pairs)
    qa = ma.gaussian_pulse(bf.lgl_operators(2)[0], (0.45, 0.5, 0.5), 0.15)
    qb = mb.gaussian_pulse(bf.lgl_operators(4)[0], (0.05, 0.5, 0.5), 0.15)
    dt = 0.5 * min(configs.stable_dt(ma, rho_a, lam_a, mu_a, 0.5),
                   configs.stable_dt(mb, rho_b, lam_b, mu_b, 0.5))
    E = [oa.energy(qa) + ob.energy(qb)]
    for _ in range(5):
        qa, qb = po.lsrk(qa, qb, dt, 3)
        E.append(oa.energy(qa) + ob.energy(qb))
    assert np.all(np.diff(E) < 0), E


# ---------------------------------------------------------------- GPU

def _gpu_pair(ma, mb, ea, eb, mats, prec=(bf.PRECISION_FP64, bf.PRECISION_FP64), flux=0):
    da = bf.GpuDomain(ma, *mats[0], bc=_glued_bc(ma), precision=prec[0], flux=flux)
    db = bf.GpuDomain(mb, *mats[1], bc=_glued_bc(mb), precision=prec[1], flux=flux)
    g = bf.PGlue(da, db, ea, eb)
    return da, db, g


GPU_CASES = [
    # dim, Na, Nb, base cells along y/z, refine, x cells per half
    (3, 3, 5, 3, 0.5, (3, 3)),
    (3, 5, 7, 2, 0.5, (3, 2)),
    (3, 2, 4, 3, 0.0, (2, 2)),
    (3, 5, 5, 2, 0.5, (3, 3)),
    (2, 3, 5, 4, 0.5, (3, 4)),
    (2, 1, 6, 3, 0.0, (2, 2)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_CASES, ids=lambda c: f"{c[0]}d-N{c[1]}-N{c[2]}")
@pytest.mark.parametrize("flux", [0, 1], ids=["upwind", "central"])
def test_gpu_glued_domains_match_the_oracle(case, flux):
    dim, Na, Nb, n, p, nx = case
    ma, mb, ea, eb, pairs = split_brick(dim, Na, Nb, n, seed=Na + Nb, refine=p, nx=nx)
    mats = [bf.material_random(ma.K, 3), bf.material_random(mb.K, 4)]
    qa = ma.gaussian_pulse(bf.lgl_operators(Na)[0], (0.4, 0.5, 0.5), 0.2)
    qb = mb.gaussian_pulse(bf.lgl_operators(Nb)[0], (0.1, 0.5, 0.5), 0.2)
    dt = min(configs.stable_dt(ma, *mats[0], 0.5), configs.stable_dt(mb, *mats[1], 0.5))
    da, db, g = _gpu_pair(ma, mb, ea, eb, mats, flux=flux)
    da.set_fields(qa)
    db.set_fields(qb)
    b = bf.Batch([da, db])
    b.add_pglue(g)
    # per stage: the glue, then each order group's levels (equal orders
    # share a group)
    lv = [da.launch_levels(), db.launch_levels()]
    lv = max(lv) if Na == Nb else sum(lv)
    assert b.launches_per_step() == 1 + 5 * (lv + 1)
    po = orc.PGlueOracle(orc.Oracle.from_mesh(ma, *mats[0], flux),
                         orc.Oracle.from_mesh(mb, *mats[1], flux), pairs)
    n0 = bf.launch_count()
    b.step(dt, 1)
    b.sync()
    assert bf.launch_count() - n0 == b.launches_per_step()
    ra, rb = po.lsrk(qa, qb, dt, 1)
    assert relerr(da.get_fields(), ra).max() < 1e-12
    assert relerr(db.get_fields(), rb).max() < 1e-12
    b.step(dt, 9)
    b.sync()
    ra, rb = po.lsrk(ra, rb, dt, 9)
    assert relerr(da.get_fields(), ra).max() < 1e-12
    assert relerr(db.get_fields(), rb).max() < 1e-12
    b.free()


@pytest.mark.gpu
def test_gpu_glue_with_a_precision_form_side():
    ma, mb, ea, eb, pairs = split_brick(3, 3, 5, 3, seed=2, refine=0.4, nx=(3, 3))
    mats = [bf.material_random(ma.K, 5), bf.material_random(mb.K, 6)]
    qa = ma.gaussian_pulse(bf.lgl_operators(3)[0], (0.3, 0.5, 0.5), 0.2)
    qb = mb.gaussian_pulse(bf.lgl_operators(5)[0], (0.2, 0.5, 0.5), 0.2)
    dt = min(configs.stable_dt(ma, *mats[0], 0.5), configs.stable_dt(mb, *mats[1], 0.5))
    da, db, g = _gpu_pair(ma, mb, ea, eb, mats,
                          prec=(bf.PRECISION_FP32, bf.PRECISION_FP64))
    da.set_fields(qa)
    db.set_fields(qb)
    b = bf.Batch([da, db])
    b.add_pglue(g)
    b.step(dt, 20)
    b.sync()
    po = orc.PGlueOracle(orc.Oracle.from_mesh(ma, *mats[0]),
                         orc.Oracle.from_mesh(mb, *mats[1]), pairs)
    ra, rb = po.lsrk(qa, qb, dt, 20)
    got = np.concatenate([da.get_fields().ravel(), db.get_fields().ravel()])
    ref = np.concatenate([ra.ravel(), rb.ravel()])
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6
    b.free()


@pytest.mark.gpu
def test_gpu_glue_checks():
    ma, mb, ea, eb, pairs = split_brick(3, 3, 5, 2, nx=(2, 2))
    mats = [(1.0, 2.0, 1.0), (1.0, 2.0, 1.0)]
    da = bf.GpuDomain(ma, *mats[0], bc=_glued_bc(ma))
    db = bf.GpuDomain(mb, *mats[1], bc=_glued_bc(mb))
    # a domain with glued faces steps only in a batch with its glue
    with pytest.raises(RuntimeError, match="glued"):
        bf.LSRK(da).step(1e-3, 1)
    with pytest.raises(RuntimeError, match="glued"):
        da.rhs()
    b = bf.Batch([da, db])
    with pytest.raises(RuntimeError, match="joined by 0 glues"):
        b.step(1e-3, 1)
    # entries that are not glued faces / glued twice / not opposite faces
    with pytest.raises(RuntimeError, match="not a glued face"):
        bf.PGlue(da, db, np.r_[ea[:-1], 10 ** 6], eb)
    with pytest.raises(RuntimeError, match="glued twice"):
        bf.PGlue(da, db, np.r_[ea[:-1], ea[0]], eb)
    half = len(ea) // 2  # the first half pairs a's +x side with b's -x side
    with pytest.raises(RuntimeError, match="opposite faces"):
        bf.PGlue(da, db, ea[:half], eb[half:])
    with pytest.raises(RuntimeError, match="glue order"):
        bf.PGlue(da, db, ea, eb, Ng=4)
    g = bf.PGlue(da, db, ea, eb)
    other = bf.Batch([da])
    with pytest.raises(RuntimeError, match="not in the batch"):
        other.add_pglue(g)
    b.add_pglue(g)
    with pytest.raises(RuntimeError, match="different times or time steps"):
        b.step([1e-3, 2e-3], 1)
    b.step(1e-3, 2)
    b.sync()
    b.free()
    other.free()


@pytest.mark.gpu
def test_gpu_glue_beside_physical_boundaries():
    """glued x sides, absorbing bottom and free-surface top (z), hanging
    faces inside both subdomains: one boundary list carries both kinds"""
    rng = np.random.default_rng(11)
    meshes = []
    for N in (3, 5):
        flags = (rng.random((3, 3, 3)) < 0.4).astype(np.uint8)  # [z][y][x]
        flags[..., 0] = 0
        flags[..., -1] = 0
        meshes.append(bf.Mesh(3, N, (3, 3, 3), L=(0.5, 1.0, 1.0),
                              refine_flags=flags.reshape(-1),
                              periodic=(False, True, False)))
    ma, mb = meshes
    ea, eb = bf.glued_x_pairs(ma, mb)
    pairs = np.stack([ma.EToEb[ea], ma.EToFb[ea], mb.EToEb[eb], mb.EToFb[eb]], axis=1)
    bc = (bf.BC_GLUED, bf.BC_GLUED, 0, 0, bf.BC_ABSORBING, bf.BC_FREE_SURFACE)
    mats = [bf.material_random(ma.K, 7), bf.material_random(mb.K, 8)]
    qa = ma.gaussian_pulse(bf.lgl_operators(3)[0], (0.4, 0.5, 0.2), 0.2)
    qb = mb.gaussian_pulse(bf.lgl_operators(5)[0], (0.1, 0.5, 0.8), 0.2)
    dt = min(configs.stable_dt(ma, *mats[0], 0.5), configs.stable_dt(mb, *mats[1], 0.5))
    da = bf.GpuDomain(ma, *mats[0], bc=bc)
    db = bf.GpuDomain(mb, *mats[1], bc=bc)
    da.set_fields(qa)
    db.set_fields(qb)
    b = bf.Batch([da, db])
    b.add_pglue(bf.PGlue(da, db, ea, eb))
    b.step(dt, 10)
    b.sync()
    po = orc.PGlueOracle(orc.Oracle.from_mesh(ma, *mats[0], bc=bc),
                         orc.Oracle.from_mesh(mb, *mats[1], bc=bc), pairs)
    ra, rb = po.lsrk(qa, qb, dt, 10)
    assert relerr(da.get_fields(), ra).max() < 1e-12
    assert relerr(db.get_fields(), rb).max() < 1e-12
    b.free()


def _pw_error_2d(Na, Nb, n, T=0.05):
    ma, mb, ea, eb, pairs = split_brick(2, Na, Nb, n, nx=(n // 2, n // 2))
    po = orc.PGlueOracle(orc.Oracle.from_mesh(ma, 1.0, 2.0, 1.0),
                         orc.Oracle.from_mesh(mb, 1.0, 2.0, 1.0), pairs)
    dt0 = min(configs.stable_dt(m, 1.0, 2.0, 1.0, 0.25) for m in (ma, mb))
    steps = int(math.ceil(T / dt0))
    qa, qb = po.lsrk(_plane_wave(ma, 0.0, 0.0), _plane_wave(mb, 0.5, 0.0), T / steps, steps)
    ea_, eb_ = _plane_wave(ma, 0.0, T), _plane_wave(mb, 0.5, T)
    num = ((qa - ea_) ** 2).sum() + ((qb - eb_) ** 2).sum()
    return math.sqrt(num / ((ea_ ** 2).sum() + (eb_ ** 2).sum()))


def test_2d_plane_wave_through_glue_of_orders_2_and_4_converges():
    """rate of the lower order (N + 1 = 3), and below order 2 everywhere"""
    e1 = _pw_error_2d(2, 4, 8)
    e2 = _pw_error_2d(2, 4, 16)
    assert math.log2(e1 / e2) > 2.7, (e1, e2)
    assert e2 < 0.7 * _pw_error_2d(2, 2, 16)
