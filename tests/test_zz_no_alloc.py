"""The allocation-free energy entry point, bfam_gpu_domain_energy_noalloc.

It exists for callers that cannot allocate device memory while a solve is
running -- a process that has committed all of the device's memory to its own
pool, or a diagnostic hook between another code's time steps.  It uses a fixed
scratch array compiled into the library instead of cudaMalloc.  This file is
named so that pytest collects it last.
"""
from __future__ import annotations

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_noalloc_energy_matches_allocating_entry_point_twice():
    m = bf.Mesh(3, 3, (4, 4, 4), refine_prob=0.3, seed=0)
    rho, lam, mu = bf.material_random(m.K, 0)
    r = bf.lgl_operators(3)[0]
    dom = bf.GpuDomain(m, rho, lam, mu)
    dom.set_fields(m.gaussian_pulse(r, (0.5, 0.5, 0.5), 0.2))
    ref = dom.energy()
    # two calls in a row share the scratch array: both must match
    for _ in range(2):
        got = dom.energy_noalloc()
        assert abs(got - ref) <= TOL * abs(ref)
    # a different state afterwards: the scratch keeps no stale contribution
    bf.LSRK(dom).step(configs.stable_dt(m, rho, lam, mu, 0.5), 3)
    ref2 = dom.energy()
    assert abs(ref2 - ref) > 1e-6 * ref  # the state really changed
    for _ in range(2):
        got = dom.energy_noalloc()
        assert abs(got - ref2) <= TOL * abs(ref2)


def test_noalloc_energy_matches_on_2d_domain():
    m = bf.Mesh(2, 4, (16, 16))
    r = bf.lgl_operators(4)[0]
    dom = bf.GpuDomain(m, 1.0, 2.0, 1.0)
    dom.set_fields(m.plane_wave(r, (2 * np.pi, 2 * np.pi), 1.0, 1.0, 2.0, 1.0))
    ref = dom.energy()
    for _ in range(2):
        assert abs(dom.energy_noalloc() - ref) <= TOL * abs(ref)


def test_noalloc_energy_rejects_domains_above_the_limit():
    # 513 x 512 = 262656 elements > BFAM_GPU_NOALLOC_MAX_ELEMENTS = 262144
    m = bf.Mesh(2, 1, (513, 512))
    assert m.K > 262144
    dom = bf.GpuDomain(m, 1.0, 2.0, 1.0)
    with pytest.raises(bf.BfamGpuError) as ei:
        dom.energy_noalloc()
    assert ei.value.code == -1
    assert "BFAM_GPU_NOALLOC_MAX_ELEMENTS" in str(ei.value)
    # the allocating entry point still works on the same domain
    assert dom.energy() == 0.0
