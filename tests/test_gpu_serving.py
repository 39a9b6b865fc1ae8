"""Serving loop on the GPU: a Poisson stream of point-source requests through
continuous batching (chunks of 7 steps, so batches are rebuilt as requests
join and leave, and a tight device budget so that admission waits).

Bar: every request's seismograms are bitwise those of the same request
solved alone (bfam_ts_lsrk on its own domain), and within 1e-12 (FP64) or
1e-6 (precision form) relative L2 of the FP64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import serving
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _alone(r: serving.Request, precision: int) -> np.ndarray:
    mesh, rho, lam, mu, dt = serving.request_problem(r)
    d = bf.GpuDomain(mesh, rho, lam, mu, precision=precision)
    d.set_source(r.source, r.force, r.f0, r.t0)
    d.set_receivers(r.receivers, r.nsteps)
    bf.LSRK(d).step(dt, r.nsteps, use_graph=True)
    s = d.seismograms()
    d.free()
    return s


def _oracle(r: serving.Request) -> np.ndarray:
    mesh, rho, lam, mu, dt = serving.request_problem(r)
    o = orc.Oracle.from_mesh(mesh, rho, lam, mu)
    o.set_source(r.source, r.force, r.f0, r.t0)
    _, s = o.seismograms(mesh.empty_fields(), 0.0, dt, r.nsteps, r.receivers)
    return s


@pytest.mark.parametrize("precision,tol", [(bf.PRECISION_FP64, 1e-12),
                                           (bf.PRECISION_FP32, 1e-6)], ids=["fp64", "fp32"])
def test_continuous_batching_matches_alone_and_oracle(precision, tol):
    reqs = serving.poisson_requests(400.0, 10, seed=5, n_range=(3, 5),
                                    steps_range=(10, 40))
    biggest = max(serving.estimate_device_bytes(r.n, r.N) for r in reqs)
    srv = serving.Server(serving.GpuEngine(precision), budget_bytes=4 * biggest,
                         chunk=7)
    stats = srv.run(reqs, realtime=True)
    s = stats.summary()
    assert s["completed"] == len(reqs)
    assert stats.max_bytes <= 4 * biggest
    assert stats.chunks > 3
    for r in reqs:
        assert r.seismograms.shape == (r.nsteps, 16, 9)
        assert np.array_equal(r.seismograms, _alone(r, precision)), r.id
    for r in sorted(reqs, key=lambda r: r.n ** 3 * r.nsteps)[:3]:
        ref = _oracle(r)
        assert np.abs(ref).max() > 0
        e = np.sqrt(((r.seismograms - ref) ** 2).sum() / (ref ** 2).sum())
        assert e < tol, (r.id, e)
