"""The CUDA path on bfam's own split of multi-level adapted bricks, against the
oracle (GPU).

Meshes come from the reference's front end compiled from source
(oracle/bfam_ref.py: p4est brick, seeded refinement passes, 2:1 balance,
bfam_domain_pxest_split_dgx_subdomains): several refinement levels, hanging
faces between adjacent levels, elements that are fine on one face and coarse
on another, bounded and periodic bricks.  Two routes into the product:
  * bfam's arrays and operators handed to the bfam_gpu C-ABI (ctypes);
  * a C program compiled against the reference's src/bfam.h that goes through
    the header-only adapter include/bfam_gpu_bfam.h on the bfam domain
    itself (tests/c/bfam_adapter_test.c).
The oracle takes only the element boxes (its neighbours come from geometry).
Bar: plain FP64 form 1e-12 relative L2 per field for the right-hand side and
the state after K LSRK steps; FP32 right-hand side 1e-6.
"""
from __future__ import annotations

import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import configs
from oracle import bfam_ref as br
from oracle import oracle as orc
from conftest import relerr

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (br.available(2) and br.available(3)),
                                 reason="oracle/_ref/libbfam_ref{2,3}d.so not built")]

TOL = 1e-12
TOL32 = 1e-6
STEPS = 10

CASES = [
    # dim, base cells, N, seed, levels, prob, periodic, bc
    (2, (4, 4), 3, 1, 3, 0.35, (1, 1), 0),
    (2, (5, 4), 5, 2, 2, 0.4, (1, 0), 1),
    (3, (3, 3, 3), 3, 1, 2, 0.35, (1, 1, 1), 0),
    (3, (3, 3, 3), 2, 2, 3, 0.3, (1, 1, 1), 0),
    (3, (2, 2, 2), 5, 3, 2, 0.3, (1, 1, 1), 0),
    (3, (2, 3, 2), 3, 4, 2, 0.4, (0, 1, 0), 1),
    (3, (2, 2, 2), 7, 6, 2, 0.2, (1, 1, 1), 0),
]


def _ids(c):
    return f"{c[0]}d-{c[1]}-N{c[2]}-L{c[4]}-per{''.join(map(str, c[6]))}"


def _problem(case):
    dim, n, N, seed, levels, prob, per, bc = case
    m = br.BfamMesh(dim, n, N, seed=seed, levels=levels, prob=prob, periodic=per)
    rho, lam, mu = bf.material_random(m.K, seed + 30)
    o = orc.Oracle(dim, N, m.ecoord, m.nbase, m.L, rho, lam, mu, 0, fine=m.fine)
    if not all(per[:dim]):
        o.set_boundary(per, bc)
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((m.nfields, m.K * m.Np))
    dt = configs.stable_dt(m, rho, lam, mu, 0.4)
    return m, rho, lam, mu, o, q, dt


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_bfam_arrays_through_the_c_abi(case):
    m, rho, lam, mu, o, q, dt = _problem(case)
    bc = case[7]
    dom = bf.GpuDomain(m, rho, lam, mu, bc=bc)
    assert dom.launch_levels() >= 2
    dom.set_fields(q)
    assert relerr(dom.rhs(), o.rhs(q)).max() < TOL
    ts = bf.LSRK(dom)
    ts.step(dt, STEPS, use_graph=True)
    assert relerr(dom.get_fields(), o.lsrk(q, dt, STEPS)).max() < TOL
    ts.free()
    dom.free()


@pytest.mark.parametrize("case", [CASES[0], CASES[3], CASES[5]], ids=_ids)
def test_bfam_arrays_device_geometry_and_precision(case):
    m, rho, lam, mu, o, q, dt = _problem(case)
    bc = case[7]
    host = bf.GpuDomain(m, rho, lam, mu, bc=bc)
    dev = bf.GpuDomain(m, rho, lam, mu, bc=bc, geometry="device")
    x0h, hh = host.geometry()
    x0d, hd = dev.geometry()
    assert np.array_equal(x0h, x0d) and np.array_equal(hh, hd)
    host.free()
    dev.free()
    f32 = bf.GpuDomain(m, rho, lam, mu, bc=bc, precision=bf.PRECISION_FP32)
    f32.set_fields(q)
    ts = bf.LSRK(f32)
    ts.step(dt, STEPS)
    assert relerr(f32.get_fields(), o.lsrk(q, dt, STEPS)).max() < TOL32
    ts.free()
    f32.free()


ADAPTER = [
    # case index, geometry (0: node coordinate fields, 1: quadrants)
    (0, 0), (1, 1), (3, 0), (4, 1), (5, 0),
]


def _run_adapter(case, geometry, tmp: Path):
    dim, n, N, seed, levels, prob, per, bc = case
    m, rho, lam, mu, o, q, dt = _problem(case)
    exe = br.REF / f"bfam_adapter_test{dim}d"
    if not exe.exists():
        pytest.skip(f"{exe} not built")
    nn = list(n) + [1] * (3 - len(n))
    pp = list(per) + [1] * (3 - len(per))
    hdr = [0x62666164, dim, N, *nn, *pp, levels, seed, STEPS, 0, 0, geometry, bc]
    fin, fout = tmp / "in.bin", tmp / "out.bin"
    with open(fin, "wb") as f:
        f.write(struct.pack("16i", *hdr))
        f.write(struct.pack("5d", prob, 1.0, 1.0, 1.0, dt))
        f.write(struct.pack("i", m.K))
        f.write(np.concatenate([rho, lam, mu]).astype(np.float64).tobytes())
        f.write(np.ascontiguousarray(q).tobytes())
    r = subprocess.run([str(exe), str(fin), str(fout)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = fout.read_bytes()
    status, K, aux, checks = struct.unpack("4i", raw[:16])
    assert (status, K) == (0, m.K)
    body = np.frombuffer(raw[16:], dtype=np.float64).reshape(2, m.nfields, -1)
    return m, o, q, dt, aux, checks, body[0], body[1]


@pytest.mark.parametrize("entry", ADAPTER,
                         ids=lambda e: _ids(CASES[e[0]]) + ("-quads" if e[1] else "-grid"))
def test_c_adapter_on_bfam_domain(entry, tmp_path):
    case = CASES[entry[0]]
    m, o, q, dt, aux, checks, rhs, qn = _run_adapter(case, entry[1], tmp_path)
    assert aux == 1      # aux_rates called once, on the one volume subdomain
    assert checks == 5   # bad field list refused, upload, rates, download, push
    assert relerr(rhs, o.rhs(q)).max() < TOL
    assert relerr(qn, o.lsrk(q, dt, STEPS)).max() < TOL
