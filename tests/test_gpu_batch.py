"""Batches of domains, point sources and receivers, through the bfam_gpu
C-ABI.

Bar: a domain stepped inside a batch is bitwise the same as the domain
stepped alone (the per-element arithmetic is the same code); the FP64 plain
form agrees with the FP64 oracle to 1e-12 relative L2 per field, and so do
its receiver seismograms; the precision form's seismograms to 1e-6."""
from __future__ import annotations

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from oracle import oracle as orc
from conftest import relerr

pytestmark = pytest.mark.gpu

# dim, N, base cells, refine prob, seed, precision
MIX = [
    (3, 3, (4, 4, 4), 0.3, 1, bf.PRECISION_FP64),
    (3, 5, (3, 3, 3), 0.3, 2, bf.PRECISION_FP64),
    (3, 7, (2, 2, 2), 0.5, 3, bf.PRECISION_FP64),
    (3, 5, (2, 3, 2), 0.4, 4, bf.PRECISION_FP32),
    (3, 5, (3, 2, 2), 0.2, 5, bf.PRECISION_FP64),
    (2, 4, (6, 5), 0.4, 6, bf.PRECISION_FP64),
]


def _problem(dim, N, n, p, seed, prec):
    m = bf.Mesh(dim, N, n, refine_prob=p, seed=seed)
    rho, lam, mu = bf.material_random(m.K, seed + 7)
    r = bf.lgl_operators(N)[0]
    q0 = m.gaussian_pulse(r, (0.5, 0.5, 0.5), 0.2)
    dt = configs.stable_dt(m, rho, lam, mu, 0.5)
    return m, rho, lam, mu, q0, dt


def _alone(m, rho, lam, mu, q0, dt, nsteps, prec, src=None, recv=None):
    d = bf.GpuDomain(m, rho, lam, mu, precision=prec)
    d.set_fields(q0)
    if src:
        d.set_source(*src)
    if recv is not None:
        d.set_receivers(recv, nsteps)
    bf.LSRK(d).step(dt, nsteps, use_graph=True)
    out = d.get_fields(), (d.seismograms() if recv is not None else None)
    d.free()
    return out


def test_batch_equals_each_domain_alone_and_the_oracle():
    probs = [_problem(*c) for c in MIX]
    doms = []
    for (m, rho, lam, mu, q0, dt), c in zip(probs, MIX):
        d = bf.GpuDomain(m, rho, lam, mu, precision=c[5])
        d.set_fields(q0)
        doms.append(d)
    b = bf.Batch(doms)
    groups = b.groups()
    # (3,3) (3,5,fp64) (3,7) (3,5,fp32) (2,4): two fp64 N=5 domains share a group
    assert len(groups) == 5
    assert sum(g["elements"] for g in groups) == sum(p[0].K for p in probs)
    dts = [p[5] for p in probs]
    nsteps = 6
    n0 = bf.launch_count()
    b.step(dts, nsteps)
    b.sync()
    per_step = b.launches_per_step()
    # one launch per order group, refinement level and stage, plus post-step
    lv = [d.launch_levels() for d in doms]
    assert all(x == 2 for x in lv)  # every mesh here has hanging faces
    assert per_step == 1 + 5 * 2 * len(groups)
    assert bf.launch_count() - n0 == nsteps * per_step
    for i, ((m, rho, lam, mu, q0, dt), c) in enumerate(zip(probs, MIX)):
        got = doms[i].get_fields()
        alone, _ = _alone(m, rho, lam, mu, q0, dt, nsteps, c[5])
        assert np.array_equal(got, alone), i
        assert abs(b.time(i) - nsteps * dt) < 1e-15
        if c[5] == bf.PRECISION_FP64:
            ref = orc.Oracle.from_mesh(m, rho, lam, mu).lsrk(q0, dt, nsteps)
            assert relerr(got, ref).max() < 1e-12, i
    b.free()


def test_batch_graph_equals_eager_and_steps_continue():
    probs = [_problem(*c) for c in MIX[:3]]
    res = []
    for use_graph in (False, True):
        doms = []
        for m, rho, lam, mu, q0, dt in probs:
            d = bf.GpuDomain(m, rho, lam, mu)
            d.set_fields(q0)
            doms.append(d)
        b = bf.Batch(doms)
        dts = [p[5] for p in probs]
        b.step(dts, 3, use_graph=use_graph)
        b.step(dts, 4, use_graph=use_graph)  # odd parity after 3 steps
        res.append([d.get_fields() for d in doms])
        b.free()
    for a, c in zip(*res):
        assert np.array_equal(a, c)


def test_every_tile_gives_the_same_result():
    """every compiled tile -- one element per CTA with any register budget,
    several elements per CTA, one warp per element -- steps bitwise alike"""
    cases = [(3, 3, (4, 4, 4), 0.3, 1, 0), (3, 5, (3, 3, 3), 0.3, 2, 0),
             (3, 7, (2, 2, 2), 0.5, 3, 0), (3, 5, (3, 3, 3), 0.3, 2, 1),
             (3, 1, (3, 3, 3), 0.4, 4, 0), (3, 2, (3, 2, 3), 0.4, 5, 0),
             (3, 3, (3, 3, 3), 0.5, 6, 1), (3, 4, (2, 3, 2), 0.5, 7, 0)]
    for c in cases:
        m, rho, lam, mu, q0, dt = _problem(*c)
        out = []
        for tile in range(len(bf.tile_shapes(3, c[1]))):
            for cps in (0, 1):
                d = bf.GpuDomain(m, rho, lam, mu, precision=c[5])
                d.set_fields(q0)
                b = bf.Batch([d])
                b.set_tile(0, tile, cps)
                b.step([dt], 4)
                out.append(d.get_fields())
                b.free()
                d.free()
        for o in out[1:]:
            assert np.array_equal(o, out[0]), c


def _receivers(rng, n):
    return rng.uniform(0.05, 0.95, size=(n, 3))


@pytest.mark.parametrize("prec,tol", [(bf.PRECISION_FP64, 1e-12), (bf.PRECISION_FP32, 1e-6)],
                         ids=["fp64", "fp32"])
def test_point_source_and_receivers_against_the_oracle(prec, tol):
    m, rho, lam, mu, _, dt = _problem(3, 4, (3, 3, 3), 0.3, 11, prec)
    q0 = m.empty_fields()
    rng = np.random.default_rng(4)
    recv = _receivers(rng, 16)
    src = ((0.41, 0.57, 0.33), (0.3, -0.2, 1.0), 10.0, 0.1)
    nsteps = 60
    q, seis = _alone(m, rho, lam, mu, q0, dt, nsteps, prec, src, recv)
    o = orc.Oracle.from_mesh(m, rho, lam, mu)
    o.set_source(*src)
    qr, sr = o.seismograms(q0, 0.0, dt, nsteps, recv)
    assert seis.shape == (nsteps, 16, 9)
    assert np.abs(sr).max() > 1e-6  # the wave reached the receivers
    assert relerr(q, qr).max() < tol
    e = np.sqrt(((seis - sr) ** 2).sum()) / np.sqrt((sr ** 2).sum())
    assert e < tol, e


def test_sources_alone_and_in_the_mix_are_identical():
    rng = np.random.default_rng(9)
    cases = [(3, 3, (3, 3, 3), 0.3, 21, 0), (3, 5, (2, 2, 2), 0.5, 22, 0),
             (3, 5, (2, 2, 3), 0.3, 23, 1)]
    probs, srcs, recvs, doms = [], [], [], []
    nsteps = 25
    for c in cases:
        m, rho, lam, mu, _, dt = _problem(*c)
        q0 = m.empty_fields()
        src = (tuple(rng.uniform(0.1, 0.9, 3)), tuple(rng.normal(size=3)),
               rng.uniform(5, 15), 0.08)
        recv = _receivers(rng, 16)
        d = bf.GpuDomain(m, rho, lam, mu, precision=c[5])
        d.set_fields(q0)
        d.set_source(*src)
        d.set_receivers(recv, nsteps)
        probs.append((m, rho, lam, mu, q0, dt))
        srcs.append(src)
        recvs.append(recv)
        doms.append(d)
    b = bf.Batch(doms)
    b.step([p[5] for p in probs], nsteps)
    b.sync()
    for i, c in enumerate(cases):
        m, rho, lam, mu, q0, dt = probs[i]
        q, seis = _alone(m, rho, lam, mu, q0, dt, nsteps, c[5], srcs[i], recvs[i])
        assert np.array_equal(doms[i].get_fields(), q)
        assert np.array_equal(doms[i].seismograms(), seis)
    b.free()


def test_receivers_stop_at_max_samples_and_clock_keeps_time():
    m, rho, lam, mu, q0, dt = _problem(3, 3, (2, 2, 2), 0.0, 1, 0)
    d = bf.GpuDomain(m, rho, lam, mu)
    d.set_fields(q0)
    d.set_receivers(np.array([[0.3, 0.3, 0.3]]), 5)
    ts = bf.LSRK(d)
    ts.step(dt, 8, use_graph=True)
    s = d.seismograms()
    assert s.shape == (5, 1, 9)
    o = orc.Oracle.from_mesh(m, rho, lam, mu)
    _, sr = o.seismograms(q0, 0.0, dt, 5, np.array([[0.3, 0.3, 0.3]]))
    assert np.abs(s - sr).max() <= 1e-12 * np.abs(sr).max()


def test_source_outside_the_mesh_is_rejected():
    m, rho, lam, mu, q0, dt = _problem(3, 3, (2, 2, 2), 0.0, 1, 0)
    d = bf.GpuDomain(m, rho, lam, mu)
    with pytest.raises(bf.BfamGpuError) as ei:
        d.set_source((1.5, 0.5, 0.5), (1, 0, 0), 10.0, 0.1)
    assert ei.value.code == bf.BFAM_GPU_EINVAL
    with pytest.raises(bf.BfamGpuError):
        d.set_receivers(np.array([[0.5, -0.1, 0.5]]), 4)


def test_elements_per_cta_tiles_across_domains():
    """a CTA's elements may belong to different domains (uneven counts, so
    that CTAs straddle domain boundaries and the last CTA is partly empty):
    each domain equals itself stepped alone and the oracle"""
    meshes = [bf.Mesh(3, 3, n, refine_prob=0.4, seed=s)
              for n, s in (((3, 3, 3), 11), ((2, 3, 2), 12), ((1, 1, 3), 13))]
    probs = []
    for k, m in enumerate(meshes):
        rho, lam, mu = bf.material_random(m.K, 20 + k)
        q0 = np.random.default_rng(k).standard_normal((m.nfields, m.K * m.Np))
        probs.append((m, rho, lam, mu, q0))
    dt = min(configs.stable_dt(m, r, l, u, 0.4) for m, r, l, u, _ in probs)
    epc = bf.tile_elements(3, 3)
    for tile in [t for t, e in enumerate(epc) if e > 1]:
        doms = []
        for m, rho, lam, mu, q0 in probs:
            d = bf.GpuDomain(m, rho, lam, mu)
            d.set_fields(q0)
            doms.append(d)
        b = bf.Batch(doms)
        b.set_tile(0, tile, 0)
        b.step([dt] * len(doms), 3)
        for d, (m, rho, lam, mu, q0) in zip(doms, probs):
            ref = orc.Oracle.from_mesh(m, rho, lam, mu).lsrk(q0, dt, 3)
            assert relerr(d.get_fields(), ref).max() < 1e-12, (tile, m.K)
        b.free()
        for d in doms:
            d.free()
