"""Benchmark problems for the DG elastic hot path (synthetic, seeded).

Each builder returns a Problem: a brick mesh in bfam's data model, per-element
material, initial state, time step and step count.  All random draws use the
PCG32 stream of the reference (refinement: stream 1, material: stream 2,
elements visited in Morton order).

  cfg0  2D, 16x16 periodic conforming brick, N=4, rho=1 lambda=2 mu=1,
        P plane wave k=(2pi,2pi), KC54, CFL 0.5, 100 steps
  cfg1  3D, 32^3 periodic brick, each base cell refined once with p=0.3
        (seed 0), N=5, rho~U[1,3], cp~U[4,6], cs=cp/U[1.6,2.0], Gaussian
        pressure pulse width 0.05 at the centre, 200 steps
  cfg2  cfg1's mesh and material at N=7 (heterogeneous, for throughput and
        error against the FP64 path); homogeneous variant with the plane wave
        k=(2pi,0,0) for the analytic error over one period
  cfg3  256 independent 3D instances: final element count K drawn
        log-uniform in [512, 32768] (seed 1), order from {3, 5, 7}, base
        brick of about K / 2.4 cells refined once with p = 0.2, cfg1's
        material law and a Gaussian pulse; precision form
Time step: dt = CFL * min_e(min_a h_{e,a} / cp_e) / N^2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import PCG32, Mesh, lgl_operators, material_random


@dataclass
class Problem:
    name: str
    mesh: Mesh
    rho: np.ndarray
    lam: np.ndarray
    mu: np.ndarray
    q0: np.ndarray
    dt: float
    nsteps: int
    meta: dict = field(default_factory=dict)

    @property
    def ndof(self) -> int:
        return self.mesh.ndof


def stable_dt(mesh: Mesh, rho, lam, mu, cfl: float) -> float:
    rho = np.broadcast_to(rho, (mesh.K,))
    cp = np.sqrt((np.broadcast_to(lam, (mesh.K,)) + 2 * np.broadcast_to(mu, (mesh.K,))) / rho)
    hmin = mesh.h[:, :mesh.dim].min(axis=1)
    return float(cfl * np.min(hmin / cp) / (mesh.N * mesh.N))


def cfg0() -> Problem:
    N = 4
    mesh = Mesh(2, N, (16, 16))
    r = lgl_operators(N)[0]
    rho, lam, mu = (np.full(mesh.K, v) for v in (1.0, 2.0, 1.0))
    q0 = mesh.plane_wave(r, (2 * math.pi, 2 * math.pi), 1.0, 1.0, 2.0, 1.0, 0.0)
    dt = stable_dt(mesh, rho, lam, mu, 0.5)
    return Problem("cfg0", mesh, rho, lam, mu, q0, dt, 100,
                   {"k": (2 * math.pi, 2 * math.pi), "amplitude": 1.0})


def heterogeneous_brick(N: int, n: int = 32, refine_prob: float = 0.3, seed: int = 0,
                        width: float = 0.05, nsteps: int = 200, cfl: float = 0.5,
                        name: str = "cfg1", dims=None) -> Problem:
    mesh = Mesh(3, N, dims or (n, n, n), refine_prob=refine_prob, seed=seed)
    r = lgl_operators(N)[0]
    rho, lam, mu = material_random(mesh.K, seed)
    q0 = mesh.gaussian_pulse(r, (0.5, 0.5, 0.5), width)
    dt = stable_dt(mesh, rho, lam, mu, cfl)
    return Problem(name, mesh, rho, lam, mu, q0, dt, nsteps,
                   {"n": n, "refine_prob": refine_prob, "seed": seed, "width": width})


def cfg1(n: int = 32, nsteps: int = 200) -> Problem:
    return heterogeneous_brick(5, n=n, nsteps=nsteps, name="cfg1")


def cfg2(n: int = 32, nsteps: int = 200) -> Problem:
    return heterogeneous_brick(7, n=n, nsteps=nsteps, name="cfg2")


def plane_wave_3d(N: int, n: int, refine_prob: float = 0.3, seed: int = 0,
                  cfl: float = 0.5, periods: float = 1.0) -> Problem:
    """Homogeneous rho=1, lambda=2, mu=1 (cp=2) P wave k=(2pi,0,0); one period
    is T = 2pi / (cp |k|) = 0.5."""
    mesh = Mesh(3, N, (n, n, n), refine_prob=refine_prob, seed=seed)
    r = lgl_operators(N)[0]
    rho, lam, mu = (np.full(mesh.K, v) for v in (1.0, 2.0, 1.0))
    k = (2 * math.pi, 0.0, 0.0)
    q0 = mesh.plane_wave(r, k, 1.0, 1.0, 2.0, 1.0, 0.0)
    T = periods * 0.5
    dt0 = stable_dt(mesh, rho, lam, mu, cfl)
    nsteps = int(math.ceil(T / dt0))
    return Problem(f"plane_wave_N{N}_n{n}", mesh, rho, lam, mu, q0, T / nsteps, nsteps,
                   {"k": k, "T": T})


def cfg3_specs(count: int = 256, seed: int = 1, orders=(3, 5, 7), kmin: int = 512,
               kmax: int = 32768, refine_prob: float = 0.2) -> list[dict]:
    """Instance draws of the batching workload (PCG32 seed `seed`, stream 3):
    K log-uniform in [kmin, kmax] is the target final element count; the
    base brick has about K / (1 + 7 p) cells, as close to a cube as whole
    cells allow."""
    g = PCG32(seed, 3)
    out = []
    for i in range(count):
        u = g.uniform()
        K = math.exp(math.log(kmin) + u * (math.log(kmax) - math.log(kmin)))
        N = orders[g.bounded(len(orders))]
        base = K / (1 + 7 * refine_prob)
        nx = max(1, round(base ** (1.0 / 3.0)))
        nz = max(1, round(base / (nx * nx)))
        out.append({"index": i, "N": N, "n": (nx, nx, nz), "K_target": K,
                    "refine_prob": refine_prob, "seed": seed * 100000 + i})
    return out


def cfg3_instance(spec: dict, width: float = 0.05, cfl: float = 0.5,
                  nsteps: int = 100) -> Problem:
    p = heterogeneous_brick(spec["N"], n=1, refine_prob=spec["refine_prob"],
                            seed=spec["seed"], width=width, nsteps=nsteps, cfl=cfl,
                            name=f"cfg3[{spec['index']}]", dims=spec["n"])
    p.meta.update(spec)
    return p
