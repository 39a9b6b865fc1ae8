"""Scheduling logic of the serving loop, on the CPU with a stand-in engine:
admission against the device budget and the slot limit, chunking at the
shortest remaining request, retirement, latency bookkeeping."""
from __future__ import annotations

import numpy as np
import pytest

from bfam_b200 import serving


class FakeEngine:
    """Records what the server asks of the device."""

    def __init__(self):
        self.live = {}
        self.steps = []
        self.max_live = 0
        self.closed = False

    def create(self, r):
        d = object()
        self.live[id(d)] = r
        self.max_live = max(self.max_live, len(self.live))
        r.dofs = r.n ** 3 * (r.N + 1) ** 3 * 9
        return d, 1e-3 * r.N, serving.estimate_device_bytes(r.n, r.N) - 4096

    def step(self, doms, dts, times, chunk):
        for d in doms:
            r = self.live[id(d)]
            assert r.steps_done + chunk <= r.nsteps  # never past the end
        self.steps.append((len(doms), chunk))

    def wait(self):
        pass

    def retire(self, d):
        r = self.live[id(d)]
        return np.full((r.nsteps, len(r.receivers), 9), float(r.id))

    def release(self, d):
        del self.live[id(d)]

    def close(self):
        self.closed = True


def test_request_stream_is_seeded_and_in_range():
    a = serving.poisson_requests(50.0, 40, seed=2)
    b = serving.poisson_requests(50.0, 40, seed=2)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.array_equal(x.receivers, y.receivers) for x, y in zip(a, b))
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    for r in a:
        assert 8 <= r.n <= 24 and r.N in (3, 5) and 50 <= r.nsteps <= 400
        assert 5.0 <= r.f0 <= 15.0 and r.receivers.shape == (16, 3)
        assert abs(np.linalg.norm(r.force) - 1.0) < 1e-12
        assert all(0.0 <= x < 1.0 for x in r.source)
    # mean inter-arrival time close to 1/rate
    many = serving.poisson_requests(50.0, 2000, seed=3)
    gaps = np.diff([0.0] + [r.arrival for r in many])
    assert abs(gaps.mean() - 1 / 50.0) < 0.1 / 50.0


@pytest.mark.parametrize("budget_requests,max_active", [(3, 1024), (100, 2), (100, 1024)])
def test_budget_slots_chunks_and_retirement(budget_requests, max_active):
    reqs = serving.poisson_requests(1000.0, 25, seed=7, n_range=(2, 6),
                                    steps_range=(5, 40))
    biggest = max(serving.estimate_device_bytes(r.n, r.N) for r in reqs)
    eng = FakeEngine()
    srv = serving.Server(eng, budget_bytes=budget_requests * biggest,
                         max_active=max_active, chunk=7)
    stats = srv.run(reqs, realtime=False)
    assert eng.closed and not eng.live
    assert stats.max_bytes <= budget_requests * biggest
    assert stats.max_active <= max_active
    assert eng.max_live <= max_active
    for r in reqs:
        assert r.steps_done == r.nsteps
        assert r.seismograms.shape == (r.nsteps, 16, 9) and r.seismograms[0, 0, 0] == r.id
        assert r.finished >= r.admitted >= 0 and r.latency is not None
    assert all(c <= 7 for _, c in eng.steps)
    assert stats.dof_updates == sum(r.dofs * 5 * r.nsteps for r in reqs)
    s = stats.summary()
    # arrivals are not waited for here, so latencies may be negative
    assert s["completed"] == len(reqs) and s["p99_s"] >= s["p50_s"]


def test_request_larger_than_the_budget_is_rejected_up_front():
    reqs = serving.poisson_requests(10.0, 3, seed=1, n_range=(20, 24))
    with pytest.raises(ValueError):
        serving.Server(FakeEngine(), budget_bytes=10 ** 6).run(reqs, realtime=False)


def test_realtime_admission_waits_for_arrivals():
    reqs = serving.poisson_requests(200.0, 6, seed=4, n_range=(2, 3), steps_range=(3, 6))
    t = [0.0]

    def clock():
        t[0] += 1e-3
        return t[0]

    eng = FakeEngine()
    srv = serving.Server(eng, chunk=4, clock=clock, sleep=lambda s: None)
    stats = srv.run(reqs, realtime=True)
    for r in reqs:
        assert r.admitted >= r.arrival - 1e-9 and r.latency > 0
    assert stats.summary()["p99_s"] >= stats.summary()["p50_s"] > 0


def test_next_chunk_is_queued_before_new_arrivals_are_set_up():
    """after a chunk ends the server queues the next one at once and sets up
    the requests that arrived meanwhile while it runs: no set-up happens
    between a chunk's end (wait) and the next chunk's launch (step)"""
    reqs = serving.poisson_requests(1000.0, 20, seed=5, n_range=(2, 4),
                                    steps_range=(10, 30))

    class Recorder(FakeEngine):
        def __init__(self):
            super().__init__()
            self.log = []

        def create(self, r):
            self.log.append("create")
            return super().create(r)

        def step(self, doms, dts, times, chunk):
            self.log.append("step")
            return super().step(doms, dts, times, chunk)

        def wait(self):
            self.log.append("wait")

    eng = Recorder()
    serving.Server(eng, chunk=5).run(reqs, realtime=False)
    for i, ev in enumerate(eng.log):
        if ev == "wait":
            nxt = next((x for x in eng.log[i + 1:] if x != "wait"), None)
            assert nxt in ("step", None), eng.log[i:i + 4]
    assert eng.log.count("create") == len(reqs)


def test_chunks_are_cut_to_the_time_bound():
    """with max_chunk_s a chunk is cut to about that many seconds of work
    (estimated from the chunks so far), so a request admitted during a chunk
    joins within about max_chunk_s; without it chunks run the full step
    count"""
    rate = 2e10  # DOF-updates per second of the stand-in device

    def run(max_chunk_s):
        t = [0.0]
        work = []

        class Timed(FakeEngine):
            def step(self, doms, dts, times, chunk):
                super().step(doms, dts, times, chunk)
                w = sum(self.live[id(d)].dofs for d in doms) * 5
                work.append((w * chunk / rate, w / rate))
                t[0] += w * chunk / rate  # the host waits for it in wait()

        reqs = serving.poisson_requests(50.0, 30, seed=7, n_range=(8, 12),
                                        steps_range=(60, 120))
        eng = Timed()
        srv = serving.Server(eng, chunk=50, clock=lambda: t[0],
                             sleep=lambda s: None, max_chunk_s=max_chunk_s)
        srv.run(reqs, realtime=False)
        for r in reqs:
            assert r.steps_done == r.nsteps and r.finished is not None
        return work

    full = run(None)
    cut = run(0.05)
    assert max(s for s, _ in full) > 0.1
    # after the first chunk (whose time is not known yet) every chunk is at
    # most the bound, or a single step where one step exceeds it
    for chunk_s, step_s in cut[1:]:
        assert chunk_s <= 0.05 + 1e-12 or abs(chunk_s - step_s) < 1e-12
    assert len(cut) > len(full)
