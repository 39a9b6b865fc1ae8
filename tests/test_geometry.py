"""Element geometry from p4est quadrant data computed on the device
(bfam_gpu_domain_create_from_quadrants; the ID_QUAD_* layout of
src/bfam.h:1600-1606): host checks of the quadrant tables on the CPU, and on
the GPU the boxes and every result equal to the host-geometry domain's."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from test_boundary import _vol


@pytest.mark.parametrize("dim,n,L", [(2, (5, 3), (1.3, 0.7)), (3, (3, 2, 4), (1.0, 2.0, 3.0))])
def test_quadrants_reproduce_the_element_boxes(dim, n, L):
    m = bf.Mesh(dim, 2, n, L=L, refine_prob=0.5, seed=4)
    tx0, th, q, root = m.quadrants()
    assert q.shape == (m.K, bf.NQUAD) and root == (1 << (19 if dim == 3 else 30))
    assert set(np.unique(q[:, 1])) <= {0, 1}
    # every element a quadrant corner of its level
    assert (q[:, 2:2 + dim] % (root >> q[:, 1:2]) == 0).all()
    x0 = tx0[q[:, 0]] + th[q[:, 0]] * (q[:, 2:5] / root)
    h = th[q[:, 0]] * 2.0 ** -q[:, 1:2]
    assert np.array_equal(x0[:, :dim], m.x0[:, :dim])
    assert np.array_equal(h[:, :dim], m.h[:, :dim])


def _create_q(m, tx0, th, quads, root, num_trees=None):
    keep = []
    v = _vol(m, keep)
    v.x0, v.h = bf.dp(), bf.dp()
    qd = bf.QuadrantsDesc()
    qd.num_trees = len(tx0) if num_trees is None else num_trees
    qd.tree_x0, qd.tree_h = bf._dp(tx0), bf._dp(th)
    qd.quads = quads.ctypes.data_as(bf.i32p)
    qd.root_len = root
    h = C.c_void_p()
    return bf.lib().bfam_gpu_domain_create_from_quadrants(
        C.byref(v), C.byref(bf.GlueDesc()), None, C.byref(qd), C.byref(bf.Options()),
        C.byref(h))


def test_abi_rejects_bad_quadrant_tables():
    m = bf.Mesh(3, 2, (2, 2, 2))
    tx0, th, q, root = m.quadrants()
    bad = q.copy()
    bad[3, 0] = len(tx0)
    assert _create_q(m, tx0, th, bad, root) == -1 and "tree" in bf.last_error()
    bad = q.copy()
    bad[1, 1] = 20
    assert _create_q(m, tx0, th, bad, root) == -1 and "level" in bf.last_error()
    bad = q.copy()
    bad[2, 1] = 1
    bad[2, 3] = (root >> 1) + 1  # not a level-1 corner
    assert _create_q(m, tx0, th, bad, root) == -1 and "corner" in bf.last_error()
    bad = q.copy()
    bad[2, 4] = root
    assert _create_q(m, tx0, th, bad, root) == -1 and "corner" in bf.last_error()
    assert _create_q(m, tx0, th, q, root - 1) == -1 and "power of two" in bf.last_error()
    bth = th.copy()
    bth[0, 1] = 0.0
    assert _create_q(m, tx0, bth, q, root) == -1 and "tree 0" in bf.last_error()
    assert _create_q(m, tx0, th, q, root, num_trees=0) == -1
    # a NULL quadrant descriptor
    keep = []
    v = _vol(m, keep)
    h = C.c_void_p()
    rc = bf.lib().bfam_gpu_domain_create_from_quadrants(
        C.byref(v), None, None, None, C.byref(bf.Options()), C.byref(h))
    assert rc == -1 and "quads" in bf.last_error()


CASES = [
    (3, 5, (3, 3, 3), 0.3, 6, (True, True, True)),
    (3, 3, (3, 2, 4), 0.4, 4, (False, True, False)),
    (2, 4, (6, 5), 0.4, 1, (True, True)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}d-N{c[1]}")
def test_device_geometry_equals_host_geometry(case):
    dim, N, n, p, seed, periodic = case
    m = bf.Mesh(dim, N, n, L=(1.0, 1.5, 0.75)[:dim], refine_prob=p, seed=seed,
                periodic=periodic)
    rho, lam, mu = bf.material_random(m.K, seed)
    r = bf.lgl_operators(N)[0]
    q0 = m.gaussian_pulse(r, (0.4, 0.6, 0.3), 0.2)
    dt = configs.stable_dt(m, rho, lam, mu, 0.5)
    out = {}
    for geo in ("host", "device"):
        n0 = bf.launch_count()
        d = bf.GpuDomain(m, rho, lam, mu, bc=bf.BC_ABSORBING, geometry=geo)
        if geo == "device":
            assert bf.launch_count() - n0 == 1  # the geometry kernel
        x0, h = d.geometry()
        assert np.array_equal(h[:, :dim], m.h[:, :dim])
        assert np.abs(x0 - m.x0).max() <= 1e-15
        d.set_fields(q0)
        rhs = d.rhs()
        # the point source and receivers locate their elements in the
        # device-computed boxes
        d.set_source((0.37, 0.52, 0.41)[:dim], (0.0, 1.0, 0.5)[:dim], 8.0, 0.15)
        recv = np.array([[0.1, 0.2, 0.3], [0.8, 1.2, 0.6], [0.5, 0.5, 0.5]])
        d.set_receivers(recv[:, :3], 10)
        bf.LSRK(d).step(dt, 10, use_graph=True)
        out[geo] = (rhs, d.get_fields(), d.seismograms())
        d.free()
    for a, b in zip(out["host"], out["device"]):
        assert np.array_equal(a, b)
