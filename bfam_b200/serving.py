"""Serving loop: solve requests that arrive over time, batched on one GPU.

A request is a point-source solve: a periodic brick of n^3 conforming
elements, order N, a duration in LSRK steps, a Ricker point force and
receivers.  The loop keeps every admitted request's state on the device and
runs continuous batching:

  * requests that have arrived are admitted while their device bytes fit the
    HBM budget and the number of active requests is below the slot limit;
    their host-side setup (mesh, tables, upload) overlaps the GPU work in
    flight;
  * the active set advances in chunks of steps: one bfam_gpu_batch_step of
    `chunk` steps (persistent launches per order group, graph-replayed),
    never past the end of the shortest remaining request;
  * between chunks finished requests are retired (seismograms downloaded,
    device memory returned to the pool) and the requests admitted during
    the last chunk join; the batch is rebuilt with each domain's current
    time and the next chunk is queued before new arrivals are set up, so
    that the set-up overlaps the chunk on the device.

Latency of a request = completion time - arrival time, on the host clock.
The scheduling logic talks to the device through an engine object, so that
it can be exercised on the CPU with a stand-in engine.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import PCG32


@dataclass
class Request:
    id: int
    arrival: float               # seconds after the stream starts
    n: int                       # base cells per axis (n^3 elements)
    N: int                       # order
    nsteps: int
    f0: float                    # Ricker peak frequency
    t0: float                    # time of the wavelet's peak
    source: tuple                # location
    force: tuple                 # force vector
    receivers: np.ndarray        # [16][3]
    seed: int                    # material draw
    # filled in by the server
    admitted: float | None = None
    finished: float | None = None
    steps_done: int = 0
    time: float = 0.0
    seismograms: np.ndarray | None = None
    device_bytes: int = 0
    dofs: int = 0
    # latency breakdown, filled in by the server
    setup_s: float = 0.0         # host set-up of its domain (engine.create)
    joined: float | None = None  # first chunk it stepped in
    rebuilds: int = 0            # batch rebuilds while it was active
    chunks: int = 0              # chunks it stepped in

    @property
    def latency(self) -> float | None:
        return None if self.finished is None else self.finished - self.arrival


def poisson_requests(rate: float, count: int, seed: int = 2, n_range=(8, 24),
                     orders=(3, 5), steps_range=(50, 400), f0_range=(5.0, 15.0),
                     nrecv: int = 16) -> list[Request]:
    """The request stream: Poisson arrivals at `rate` per second and the
    per-request draws, all from PCG32(seed, stream 4)."""
    g = PCG32(seed, 4)
    t = 0.0
    out = []
    for i in range(count):
        t += -math.log(1.0 - g.uniform()) / rate
        n = n_range[0] + g.bounded(n_range[1] - n_range[0] + 1)
        N = orders[g.bounded(len(orders))]
        nsteps = steps_range[0] + g.bounded(steps_range[1] - steps_range[0] + 1)
        f0 = f0_range[0] + (f0_range[1] - f0_range[0]) * g.uniform()
        src = tuple(g.uniform() for _ in range(3))
        # force: unit vector uniform on the sphere
        z = 2.0 * g.uniform() - 1.0
        phi = 2.0 * math.pi * g.uniform()
        s = math.sqrt(max(0.0, 1.0 - z * z))
        force = (s * math.cos(phi), s * math.sin(phi), z)
        recv = np.array([[g.uniform() for _ in range(3)] for _ in range(nrecv)])
        out.append(Request(i, t, n, N, nsteps, f0, 1.2 / f0, src, force, recv,
                           seed * 100000 + i))
    return out


def request_problem(r: Request, cfl: float = 0.5):
    """mesh, material, time step of a request (cfg1's material law)"""
    from . import Mesh, material_random
    mesh = Mesh(3, r.N, (r.n, r.n, r.n))
    rho, lam, mu = material_random(mesh.K, r.seed)
    cp = np.sqrt((lam + 2 * mu) / rho)
    dt = cfl * float(np.min(mesh.h[:, :3].min(axis=1) / cp)) / (r.N * r.N)
    return mesh, rho, lam, mu, dt


def estimate_device_bytes(n: int, N: int) -> int:
    """device bytes of a request's domain: q twice and dq (FP64, 9 fields)
    plus per-element tables (material, face descriptors, flux constants)
    and the receivers' samples, rounded up"""
    K = n ** 3
    Np = (N + 1) ** 3
    return int(3 * 9 * K * Np * 8 + K * 320 + (1 << 20))


class GpuEngine:
    """The device side of the server: domains with sources and receivers,
    rebuilt batches, asynchronous chunks."""

    def __init__(self, precision: int, device: int = 0):
        import torch
        from . import autotune
        self.precision = precision
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        self.batch = None
        self.members = ()
        self._autotune = autotune
        self._cache = autotune.load_cache()

    def create(self, r: Request):
        from . import GpuDomain
        mesh, rho, lam, mu, dt = request_problem(r)
        d = GpuDomain(mesh, rho, lam, mu, precision=self.precision, device=self.device)
        d.set_source(r.source, r.force, r.f0, r.t0)
        d.set_receivers(r.receivers, r.nsteps)
        r.dofs = int(mesh.ndof)
        d.mesh = None
        return d, dt, d.device_bytes()

    # host time spent per kind of engine call, for the latency breakdown
    rebuilds = 0
    rebuild_s = 0.0
    launch_s = 0.0
    wait_s = 0.0

    def step(self, doms, dts, times, chunk: int) -> None:
        from . import Batch
        key = tuple(id(d) for d in doms)
        t0 = time.perf_counter()
        if self.batch is None or key != self.members:
            if self.batch is not None:
                self.batch.free()
            # each domain keeps its device clock (continuous time base)
            self.batch = Batch(doms)
            self.batch.set_stream(self.stream.cuda_stream)
            self._autotune.autotune(self.batch, cache=self._cache, device=self.device)
            self.members = key
            self.rebuilds += 1
            t1 = time.perf_counter()
            self.rebuild_s += t1 - t0
            t0 = t1
        self.batch.step(dts, chunk)
        self.launch_s += time.perf_counter() - t0

    def wait(self) -> None:
        if self.batch is not None:
            t0 = time.perf_counter()
            self.batch.sync()
            self.wait_s += time.perf_counter() - t0

    def retire(self, d) -> np.ndarray:
        s = d.seismograms()
        return s

    def release(self, d) -> None:
        if self.batch is not None and id(d) in self.members:
            self.batch.free()
            self.batch = None
            self.members = ()
        d.free()

    def close(self) -> None:
        if self.batch is not None:
            self.batch.free()
            self.batch = None


@dataclass
class ServeStats:
    requests: list
    makespan: float
    max_active: int
    max_bytes: int
    chunks: int
    dof_updates: int
    timeline: list = field(default_factory=list)
    engine_times: dict = field(default_factory=dict)

    def breakdown(self) -> dict:
        """Where the latency goes: per request the queueing (arrival to
        admission), its host set-up, the wait for the next chunk boundary
        (admission to its first chunk) and the service time (first chunk to
        completion), with the batch rebuilds and chunks it sat through; p50
        and p99 of each over the requests, and their means over the requests
        at or above the p99 latency."""
        done = [r for r in self.requests if r.latency is not None]
        if not done:
            return {}
        comp = {
            "queue_s": [r.admitted - r.arrival for r in done],
            "setup_s": [r.setup_s for r in done],
            "join_wait_s": [(r.joined if r.joined is not None else r.admitted) - r.admitted
                            for r in done],
            "service_s": [r.finished - (r.joined if r.joined is not None else r.admitted)
                          for r in done],
            "rebuilds": [r.rebuilds for r in done],
            "chunks": [r.chunks for r in done],
            "steps": [r.nsteps for r in done],
            "dofs": [r.dofs for r in done],
        }
        lat = np.array([r.latency for r in done])
        tail = lat >= np.percentile(lat, 99)
        out = {}
        for k, v in comp.items():
            a = np.asarray(v, dtype=np.float64)
            out[k] = {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
                      "tail_mean": float(a[tail].mean())}
        out["tail_latency_s"] = float(lat[tail].mean())
        out["engine"] = dict(self.engine_times)
        return out

    def summary(self) -> dict:
        lat = np.array([r.latency for r in self.requests if r.latency is not None])
        return {
            "completed": int(len(lat)),
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_s": float(lat.mean()) if len(lat) else None,
            "makespan_s": self.makespan,
            "dof_updates_per_s": self.dof_updates / self.makespan if self.makespan else None,
            "max_active": self.max_active,
            "max_device_bytes": self.max_bytes,
            "chunks": self.chunks,
            "latency_breakdown": self.breakdown(),
        }


class Server:
    """Continuous-batching request loop (see the module docstring)."""

    def __init__(self, engine, budget_bytes: int = 150 * 10 ** 9, max_active: int = 1024,
                 chunk: int = 25, clock=time.perf_counter, sleep=time.sleep,
                 max_chunk_s: float | None = None):
        """`chunk`: steps per chunk at most; `max_chunk_s`: if set, a chunk is
        also cut to about that many seconds, from the time per DOF-update of
        the chunks so far (a request admitted during a chunk waits for its
        end, so long chunks of a heavily loaded batch delay every newcomer)."""
        self.engine = engine
        self.budget = budget_bytes
        self.max_active = max_active
        self.chunk = chunk
        self.clock = clock
        self.sleep = sleep
        self.max_chunk_s = max_chunk_s

    def run(self, requests: list[Request], realtime: bool = True) -> ServeStats:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        active = []        # (request, domain, dt) stepping on the device
        joining = []       # admitted, waiting for the next chunk boundary
        used = 0
        max_used = 0
        max_act = 0
        chunks = 0
        dof_updates = 0
        in_flight = 0      # steps of the chunk on the device
        chunk_t0 = 0.0     # when the chunk in flight was issued
        spd = None         # seconds per DOF-update of the chunks so far
        t_start = self.clock()
        now = lambda: self.clock() - t_start  # noqa: E731
        for r in requests:
            if estimate_device_bytes(r.n, r.N) > self.budget:
                raise ValueError(f"request {r.id} can never fit the budget")
        while pending or active or joining or in_flight:
            # the chunk in flight ends: retire finished requests
            if in_flight:
                self.engine.wait()
                work = sum(r.dofs for r, _, _ in active) * 5 * in_flight
                if work > 0:
                    s_chunk = (self.clock() - chunk_t0) / work
                    spd = s_chunk if spd is None else 0.5 * (spd + s_chunk)
                chunks += 1
                keep = []
                for r, d, dt in active:
                    r.steps_done += in_flight
                    r.time += in_flight * dt
                    r.chunks += 1
                    dof_updates += r.dofs * 5 * in_flight
                    if r.steps_done >= r.nsteps:
                        r.seismograms = self.engine.retire(d)
                        self.engine.release(d)
                        r.finished = now()
                        used -= max(r.device_bytes, estimate_device_bytes(r.n, r.N))
                    else:
                        keep.append((r, d, dt))
                active = keep
                in_flight = 0
            # the next chunk goes to the device at once (with the requests
            # admitted meanwhile); new arrivals are set up while it runs
            for r, _, _ in joining:
                r.joined = now()
            active += joining
            joining = []
            max_act = max(max_act, len(active))
            if active:
                c = min(self.chunk, min(r.nsteps - r.steps_done for r, _, _ in active))
                if self.max_chunk_s and spd:
                    step_s = sum(r.dofs for r, _, _ in active) * 5 * spd
                    c = max(1, min(c, int(self.max_chunk_s / step_s)))
                chunk_t0 = self.clock()
                rb0 = getattr(self.engine, "rebuilds", 0)
                self.engine.step([d for _, d, _ in active], [dt for _, _, dt in active],
                                 [r.time for r, _, _ in active], c)
                if getattr(self.engine, "rebuilds", 0) != rb0:
                    for r, _, _ in active:
                        r.rebuilds += 1
                in_flight = c
            # admission: arrived requests, in arrival order, while they fit
            while pending and (not realtime or pending[0].arrival <= now()):
                r = pending[0]
                est = estimate_device_bytes(r.n, r.N)
                if used + est > self.budget or len(active) + len(joining) >= self.max_active:
                    break
                pending.popleft()
                tc = self.clock()
                d, dt, nbytes = self.engine.create(r)
                r.setup_s = self.clock() - tc
                r.device_bytes = nbytes
                r.admitted = now()
                used += max(nbytes, est)
                joining.append((r, d, dt))
            max_used = max(max_used, used)
            if not in_flight and not joining and pending:
                wait = pending[0].arrival - now()
                if wait > 0 and realtime:
                    self.sleep(min(wait, 0.01))
        self.engine.close()
        times = {k: getattr(self.engine, k) for k in ("rebuilds", "rebuild_s", "launch_s",
                                                      "wait_s") if hasattr(self.engine, k)}
        return ServeStats(list(requests), now(), max_act, max_used, chunks, dof_updates,
                          engine_times=times)
