#!/usr/bin/env python
"""Benchmark of the DG elastic RHS + LSRK hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config cfg1|cfg0|cfg2]

Workload (default cfg1): 3D velocity-stress elasticity, 32^3 periodic brick,
each base cell refined once with probability 0.3 (seed 0, 2:1 hanging faces
through mortars), N=5, heterogeneous material, Gaussian pressure pulse; FP64
state.  A step is one KC54 LSRK step (5 stages) over the whole mesh;
DOF-updates = DOFs x stages.  Inputs (3.2 GB of state) exceed L2 (126 MB),
so no flush is needed between steps.

Metric: DOF-updates/s (higher is better).  `value` is device-timed with the
state resident in HBM; `e2e` is one full solve through the C-ABI
(bfam_gpu_domain_set_fields from pinned host memory, 200 steps,
bfam_gpu_domain_get_fields back to the host).  Multi-GPU: independent
replicas, one per rank (the path has no exchange step on one mesh).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ALG_BYTES_PER_DOF_UPDATE = {5: 30.4}  # KC54: (24 + 4*32)/5 bytes, FP64 q and dq
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg1",
                    choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4", "next"])
    ap.add_argument("--periods", type=float, default=1.0,
                    help="cfg2: periods of the analytic plane wave")
    ap.add_argument("--rates", default="10,50,200,500",
                    help="cfg4: Poisson arrival rates (requests/s)")
    ap.add_argument("--requests", type=int, default=200, help="cfg4: requests per rate")
    ap.add_argument("--chunk", type=int, default=25, help="cfg4: steps per batch chunk")
    ap.add_argument("--chunk-s", type=float, default=0.1,
                    help="cfg4: seconds per batch chunk at most (0: steps only)")
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"],
                    help="arithmetic of the right-hand side (default: fp64; cfg3, cfg4: "
                         "fp32); with cfg2 it times that one form only, as cfg1 does")
    ap.add_argument("--instances", type=int, default=256, help="cfg3: number of instances")
    ap.add_argument("--sample", type=int, default=24,
                    help="cfg3: instances also solved alone in FP64 (plain form) for "
                         "throughput and error, and end to end")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--graph", type=int, default=1)
    ap.add_argument("--n", type=int, default=32,
                    help="base cells per axis for cfg1/cfg2 (smaller cases for profiling)")
    return ap.parse_args()


def build_problem(name, n=32):
    from bfam_b200 import configs
    if name == "cfg0":
        return configs.cfg0()
    return {"cfg1": configs.cfg1, "cfg2": configs.cfg2}[name](n=n)


def workload_desc(p):
    m = p.mesh
    return {
        "workload": f"{p.name}: {m.dim}D elastic DG N={m.N}, "
                    + ("x".join(str(x) for x in m.nbase[:m.dim]))
                    + f" periodic brick, refine p={p.meta.get('refine_prob', 0.0)}, "
                    f"K={m.K} elements, {m.Kg} glue elements, KC54 LSRK",
        "dofs": int(m.ndof),
        "elements": int(m.K),
        "order": int(m.N),
        "nsteps_solve": int(p.nsteps),
        "l2_flush": "inputs larger than L2 (state %.2f GB)" % (3 * m.ndof * 8 / 1e9),
    }


def measured_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel_key):
    """dram bytes per launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel_key:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 4 + i and r[4 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_init(backend=None):
    """One process per GPU (torchrun's environment); NCCL on GPUs, gloo
    without.  The replicas share no data: the group only times them."""
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1 and not dist.is_initialized():
        import datetime
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600), **kw)
    return ws, rank, local


def max_over_ranks(x: float, local: int = 0) -> float:
    """Max of a per-rank value (a device-timed interval) over the process
    group; the value itself on one process."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, t_max: float, ws: int) -> float:
    """Whole-job throughput of ws independent replicas: every rank's units
    over the slowest rank's time."""
    return units_per_rank * ws / t_max


def _oracle_rate(o, q, dt, ndof, threads, budget_s, min_steps=1):
    """DOF-updates/s of the oracle: whole KC54 steps until budget_s elapses."""
    t0 = time.perf_counter()
    steps = 0
    while True:
        q = o.lsrk(q, dt, 1, nthreads=threads)
        steps += 1
        if steps >= min_steps and time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return ndof * 5 * steps / el, steps, el


def cpu_baseline_sample(p, budget_s=8.0):
    """The oracle (FP64 CPU restatement) on this host's cores: whole KC54
    steps over the full mesh with every host thread (the headline `value`),
    one thread on the same mesh family at 8^3 base cells, and cfg0 (2D, N=4,
    16x16, 100 steps) in full with one thread and with every thread."""
    from bfam_b200 import configs
    from oracle import oracle as orc
    threads = orc.max_threads()
    o = orc.Oracle.from_mesh(p.mesh, p.rho, p.lam, p.mu)
    v_all, st_all, el_all = _oracle_rate(o, p.q0.copy(), p.dt, p.ndof, threads, budget_s)
    out = {"value": v_all, "unit": "DOF-updates/s", "cores": threads, "kind": "port",
           "nproc": os.cpu_count(),
           "sample": f"{st_all} KC54 step(s) over the full {p.name} mesh "
                     f"({p.ndof} DOFs), {threads} threads, {el_all:.1f} s"}
    if p.name in ("cfg1", "cfg2"):
        small = configs.heterogeneous_brick(p.mesh.N, n=8, name=f"{p.name} n=8")
        os1 = orc.Oracle.from_mesh(small.mesh, small.rho, small.lam, small.mu)
        v1, st1, el1 = _oracle_rate(os1, small.q0.copy(), small.dt, small.ndof, 1, 4.0)
        out["single_thread"] = {
            "value": v1, "unit": "DOF-updates/s", "cores": 1,
            "sample": f"{st1} KC54 step(s) over the {p.name} mesh family at 8^3 base "
                      f"cells ({small.ndof} DOFs), 1 thread, {el1:.1f} s"}
    c0 = configs.cfg0()
    o0 = orc.Oracle.from_mesh(c0.mesh, c0.rho, c0.lam, c0.mu)
    cfg0 = {}
    for nt in (1, threads):
        t0 = time.perf_counter()
        o0.lsrk(c0.q0, c0.dt, c0.nsteps, nthreads=nt)
        el = time.perf_counter() - t0
        cfg0[f"{nt}_threads"] = {"value": c0.ndof * 5 * c0.nsteps / el,
                                 "unit": "DOF-updates/s", "seconds": el}
    out["cfg0_full"] = dict(cfg0, sample=f"cfg0: {c0.nsteps} KC54 steps, {c0.ndof} DOFs")
    return out


def reference_problem(name, n=32):
    """cfg1/cfg2 built without the product library: the mesh by the
    reference's own front end compiled from source (p4est brick, seeded
    refinement, bfam_domain_pxest_split_dgx_subdomains), the material from
    the reference's PCG32 (seed 0, stream 2: three draws per element in
    element order), the Gaussian pulse at the reference's LGL nodes."""
    import math
    from types import SimpleNamespace
    from oracle import bfam_ref as br
    from oracle import oracle as orc
    N = {"cfg1": 5, "cfg2": 7}[name]
    m = br.BfamMesh(3, (n, n, n), N, seed=0, levels=1, prob=0.3)
    u = orc.ref_pcg32(0, 2, 3 * m.K).astype(np.float64).reshape(m.K, 3) / 4294967296.0
    rho = 1.0 + 2.0 * u[:, 0]
    cp = 4.0 + 2.0 * u[:, 1]
    cs = cp / (1.6 + 0.4 * u[:, 2])
    mu = rho * cs * cs
    lam = rho * (cp * cp - 2 * cs * cs)
    x, y, z = m.node_coordinates()
    pulse = np.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) / 0.05 ** 2)
    q0 = np.zeros((9, m.K * m.Np))
    q0[3:6] = -pulse
    cpe = np.sqrt((lam + 2 * mu) / rho)
    dt = float(0.5 * np.min(m.h[:, :3].min(axis=1) / cpe) / (N * N))
    mesh = SimpleNamespace(dim=3, N=N, K=m.K, Kg=m.Kg, nbase=m.nbase, L=m.L,
                           periodic=(True, True, True), ndof=m.K * m.Np * 9)
    o = orc.Oracle(3, N, m.ecoord, m.nbase, m.L, rho, lam, mu, 0, fine=m.fine)
    return SimpleNamespace(name=name, mesh=mesh, q0=q0, dt=dt, nsteps=200,
                           ndof=mesh.ndof, oracle=o, meta={"refine_prob": 0.3})


def run_reference(args):
    """The reference's CPU path for this workload: the reference has no
    elastic right-hand side, so it is the oracle's FP64 restatement on the
    reference's own mesh (built by its compiled front end), timed on every
    host thread; rank 0 only."""
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as orc
    name = args.config if args.config in ("cfg1", "cfg2") else "cfg1"
    p = reference_problem(name, args.n)
    o = p.oracle
    threads = orc.max_threads()
    q = p.q0.copy()
    # warm-up: at most one KC54 step; each timed step = one KC54 step
    for _ in range(max(0, min(args.warmup, 1))):
        q = o.lsrk(q, p.dt, 1, nthreads=threads)
    steps = max(1, min(args.steps, 2))
    t0 = time.perf_counter()
    for _ in range(steps):
        q = o.lsrk(q, p.dt, 1, nthreads=threads)
    el = time.perf_counter() - t0
    v = p.ndof * 5 * steps / el
    line = {
        "impl": "reference", "metric": "DOF-updates/s", "value": v, "unit": "DOF-updates/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": el / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_desc(p),
        "cpu_baseline": {"value": v, "unit": "DOF-updates/s", "cores": threads, "kind": "port",
                         "nproc": os.cpu_count(),
                         "sample": f"{steps} KC54 step(s) over the full mesh, built by the "
                                   "reference's own front end (the reference has no "
                                   "elastic RHS; this is the oracle's restatement)"},
        "e2e": {"value": v, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """cfg3: many independent instances in one batch (one persistent launch
    per order group and stage, graph-replayed steps, autotuned tiles)."""
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    import bfam_b200 as bf
    from bfam_b200 import autotune, configs

    prec = bf.PRECISION_FP64 if args.precision == "fp64" else bf.PRECISION_FP32
    specs = configs.cfg3_specs(count=args.instances)
    t_setup = time.perf_counter()
    doms, dts, ndofs, sample = [], [], [], []
    for sp in specs:
        p = configs.cfg3_instance(sp)
        d = bf.GpuDomain(p.mesh, p.rho, p.lam, p.mu, precision=prec, device=local)
        d.set_fields(p.q0)
        doms.append(d)
        dts.append(p.dt)
        ndofs.append(p.ndof)
        if len(sample) < args.sample:
            sample.append(p)
        else:
            del p
        d.mesh = None
    t_setup = time.perf_counter() - t_setup
    total = int(sum(ndofs))
    stream = torch.cuda.Stream(device=local)
    batch = bf.Batch(doms)
    batch.set_stream(stream.cuda_stream)
    t_tune = time.perf_counter()
    tiles = autotune.autotune(batch, device=local)
    t_tune = time.perf_counter() - t_tune
    W = max(3, args.warmup)
    batch.step(dts, W)
    batch.sync()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    n0 = bf.launch_count()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        batch.step(dts, args.steps)
        ev1.record(stream)
        ev1.synchronize()
    launches = bf.launch_count() - n0
    batch.sync()
    t_local = ev0.elapsed_time(ev1) / 1e3
    t_max = max_over_ranks(t_local, local)
    value = replica_value(total * 5 * args.steps, t_max, ws)
    peak, peak_kind = measured_peak()
    achieved = total * 5 * ALG_BYTES_PER_DOF_UPDATE[5] * args.steps / t_local / 1e9

    # the sample solved alone in the plain FP64 form: throughput, and the
    # batched form's error against it after the same steps
    plain_t, plain_dofs, errs, state_errs = 0.0, 0, [], []
    for i, p in enumerate(sample):
        d = bf.GpuDomain(p.mesh, p.rho, p.lam, p.mu, device=local)
        s2 = torch.cuda.Stream(device=local)
        d.set_stream(s2.cuda_stream)
        d.set_fields(p.q0)
        ts = bf.LSRK(d)
        ts.step(p.dt, W, use_graph=True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s2)
        ts.step(p.dt, args.steps, use_graph=True)
        e1.record(s2)
        e1.synchronize()
        plain_t += e0.elapsed_time(e1) / 1e3
        plain_dofs += p.ndof
        ref = d.get_fields()
        got = doms[i].get_fields()
        num = np.sqrt(((got - ref) ** 2).sum(axis=1))
        den = np.sqrt((ref ** 2).sum(axis=1))
        # a field that is (nearly) zero is measured against the largest field
        den = np.where(den > 1e-8 * den.max(), den, den.max())
        errs.append(float((num / den).max()))
        state_errs.append(float(np.sqrt(((got - ref) ** 2).sum() / (ref ** 2).sum())))
        ts.free()
        d.free()
    plain_value = plain_dofs * 5 * args.steps / plain_t if plain_t else None

    # end to end through the public API on the sample: upload from pinned
    # host memory, a full solve (100 steps) as one batch, download
    e2e = None
    if not args.no_e2e and sample:
        hosts, outs = [], []
        for p in sample:
            h = torch.empty(p.q0.shape, dtype=torch.float64, pin_memory=True).numpy()
            h[...] = p.q0
            hosts.append(h)
            outs.append(torch.empty(p.q0.shape, dtype=torch.float64, pin_memory=True).numpy())
        sdoms = doms[:len(sample)]
        sb = bf.Batch(sdoms)
        sb.set_stream(stream.cuda_stream)
        autotune.autotune(sb, device=local)
        nsolve = sample[0].nsteps
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for d, h in zip(sdoms, hosts):
            d.set_fields(h)
        sb.step([p.dt for p in sample], nsolve)
        for d, o in zip(sdoms, outs):
            d.get_fields(o)
        e1.record(stream)
        e1.synchronize()
        el = e0.elapsed_time(e1) / 1e3
        sdofs = sum(p.ndof for p in sample)
        nbytes = sum(h.nbytes for h in hosts)
        e2e = {"value": sdofs * 5 * nsolve / el, "unit": "DOF-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "step": f"first {len(sample)} instances: upload state, {nsolve} LSRK steps "
                       "as one batch, download state", "seconds": el}
        sb.free()

    if rank == 0:
        orders = {}
        for sp_, n in zip(specs, ndofs):
            orders.setdefault(sp_["N"], [0, 0])
            orders[sp_["N"]][0] += 1
            orders[sp_["N"]][1] += int(n)
        line = {
            "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": W,
            "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 rhs / f64 state" if prec == bf.PRECISION_FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": f"cfg3: {len(specs)} independent 3D elastic instances in "
                                   "one batch, K log-uniform in [512, 32768] (seed 1), "
                                   "N in {3,5,7}, 20% one-level refinement, KC54",
                       "instances": len(specs), "dofs": total,
                       "per_order": {f"N{k}": {"instances": v[0], "dofs": v[1]}
                                     for k, v in sorted(orders.items())},
                       "l2_flush": "inputs larger than L2 (state %.1f GB)" % (total * 24 / 1e9),
                       "parallelism": f"replicas{ws}", "cuda_graph": True,
                       "tiles": tiles, "setup_s": t_setup, "autotune_s": t_tune},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"of {peak_kind}",
                         "traffic": None,
                         "kernel": "dg_stage_batch_kernel (all order groups)"},
            "plain_fp64_alone": {"value": plain_value, "unit": "DOF-updates/s",
                                 "instances": len(sample),
                                 "speedup_of_value": value / plain_value if plain_value else None,
                                 "max_rel_l2_vs_plain_fp64": max(errs) if errs else None,
                                 "max_rel_l2_vs_plain_fp64_whole_state":
                                     max(state_errs) if state_errs else None},
            "cpu_baseline": None, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    batch.free()
    for d in doms:
        d.free()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def _field_errors(a, b):
    """per-field relative L2 of a against b; a (nearly) zero field is
    measured against the largest field's norm"""
    num = np.sqrt(((a - b) ** 2).sum(axis=1))
    den = np.sqrt((b ** 2).sum(axis=1))
    den = np.where(den > 1e-8 * den.max(), den, den.max())
    return [float(x) for x in num / den]


def run_precision(args):
    """cfg2: the precision form (FP32 right-hand side, FP64 state) at N=7 on
    cfg1's mesh: throughput against the plain FP64 form on the heterogeneous
    material, the error against FP64 after the timed steps, and one period
    of the analytic P plane wave (homogeneous material) in both forms."""
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    import bfam_b200 as bf
    from bfam_b200 import configs

    W = max(3, args.warmup)
    p = configs.cfg2(n=args.n)
    out = {}
    states = {}
    n0 = bf.launch_count()
    with ClockSampler(local) as clk:
        for name, prec in (("fp32", bf.PRECISION_FP32), ("fp64", bf.PRECISION_FP64)):
            dom = bf.GpuDomain(p.mesh, p.rho, p.lam, p.mu, precision=prec, device=local)
            stream = torch.cuda.Stream(device=local)
            dom.set_stream(stream.cuda_stream)
            dom.set_fields(p.q0)
            ts = bf.LSRK(dom)
            ts.step(p.dt, W, use_graph=True)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ts.step(p.dt, args.steps, use_graph=True)
            e1.record(stream)
            e1.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            out[name] = p.ndof * 5 * args.steps / t
            states[name] = dom.get_fields()
            ts.free()
            dom.free()
    launches = bf.launch_count() - n0
    err_het = _field_errors(states["fp32"], states["fp64"])
    err_het_state = float(np.sqrt(((states["fp32"] - states["fp64"]) ** 2).sum()
                                  / (states["fp64"] ** 2).sum()))
    del states
    # analytic plane wave over `periods` periods on the same mesh
    pw = configs.plane_wave_3d(7, args.n, periods=args.periods)
    r = bf.lgl_operators(7)[0]
    qe = pw.mesh.plane_wave(r, pw.meta["k"], 1.0, 1.0, 2.0, 1.0, pw.meta["T"])
    res = {}
    for name, prec in (("fp32", bf.PRECISION_FP32), ("fp64", bf.PRECISION_FP64)):
        dom = bf.GpuDomain(pw.mesh, pw.rho, pw.lam, pw.mu, precision=prec, device=local)
        dom.set_fields(pw.q0)
        bf.LSRK(dom).step(pw.dt, pw.nsteps, use_graph=True)
        res[name] = dom.get_fields()
        dom.free()
    names = list(bf.FIELDS_3D)
    scale = np.sqrt((qe ** 2).sum())
    plane = {
        "steps": pw.nsteps, "dt": pw.dt, "T": pw.meta["T"],
        "rel_l2_vs_analytic": {k: float(np.sqrt(((res[k] - qe) ** 2).sum()) / scale)
                               for k in res},
        "rel_l2_fp32_vs_fp64_per_field": dict(zip(names, _field_errors(res["fp32"], res["fp64"]))),
        "rel_l2_vs_analytic_per_field": {
            k: dict(zip(names, [float(np.sqrt(((res[k][f] - qe[f]) ** 2).sum()) / scale)
                                for f in range(9)])) for k in res},
        "note": "per-field errors against the analytic solution are relative to the "
                "whole state's norm (vy, vz and the shear stresses are zero)",
    }
    if rank == 0:
        peak, peak_kind = measured_peak()
        ach = p.ndof * ALG_BYTES_PER_DOF_UPDATE[5] * 5 * out["fp32"] / (p.ndof * 5) / 1e9
        line = {
            "metric": "DOF-updates/s", "value": out["fp32"], "unit": "DOF-updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": W,
            "ms_per_step": p.ndof * 5 / out["fp32"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 rhs / f64 state",
            "data": "synthetic",
            "config": dict(workload_desc(p), parallelism=f"replicas{ws}", cuda_graph=True),
            "precision_form": {
                "fp32_value": out["fp32"], "fp64_value": out["fp64"],
                "speedup_vs_plain_fp64": out["fp32"] / out["fp64"],
                "heterogeneous_rel_l2_fp32_vs_fp64_per_field": dict(zip(names, err_het)),
                "heterogeneous_rel_l2_fp32_vs_fp64_whole_state": err_het_state,
                "heterogeneous_steps": W + args.steps,
                "plane_wave": plane,
            },
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_source": f"of {peak_kind}",
                         "traffic": None,
                         "kernel": "dg_stage_kernel N=7 precision form"},
            "cpu_baseline": None, "e2e": None,
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    """cfg4: Poisson streams of point-source requests through the
    continuous-batching server, one run per arrival rate."""
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    import bfam_b200 as bf
    from bfam_b200 import autotune, serving
    from oracle import oracle as orc

    prec = bf.PRECISION_FP64 if args.precision == "fp64" else bf.PRECISION_FP32
    # tile choices for the request orders, before any clock starts
    for N in (3, 5):
        m = bf.Mesh(3, N, (8, 8, 8))
        d = bf.GpuDomain(m, 1.0, 2.0, 1.0, precision=prec, device=local)
        b = bf.Batch([d])
        autotune.autotune(b, device=local)
        b.free()
        d.free()
    runs = []
    checks = []
    n0 = bf.launch_count()
    with ClockSampler(local) as clk:
        for rate in [float(x) for x in args.rates.split(",")]:
            reqs = serving.poisson_requests(rate, args.requests, seed=2)
            srv = serving.Server(serving.GpuEngine(prec, device=local),
                                 budget_bytes=150 * 10 ** 9, chunk=args.chunk,
                                 max_chunk_s=args.chunk_s or None)
            stats = srv.run(reqs, realtime=True)
            s = stats.summary()
            s["rate_per_s"] = rate
            s["requests"] = len(reqs)
            runs.append(s)
            # accuracy: the smallest requests against the FP64 oracle; one
            # request re-solved alone on the GPU must match bitwise
            for r in sorted(reqs, key=lambda r: r.n ** 3 * (r.N + 1) ** 3 * r.nsteps)[:2]:
                mesh, rho, lam, mu, dt = serving.request_problem(r)
                o = orc.Oracle.from_mesh(mesh, rho, lam, mu)
                o.set_source(r.source, r.force, r.f0, r.t0)
                _, ref = o.seismograms(mesh.empty_fields(), 0.0, dt, r.nsteps, r.receivers,
                                       nthreads=orc.max_threads())
                e = float(np.sqrt(((r.seismograms - ref) ** 2).sum() / (ref ** 2).sum()))
                checks.append({"rate": rate, "request": r.id, "n": r.n, "N": r.N,
                               "steps": r.nsteps, "rel_l2_vs_fp64_oracle": e})
            r = reqs[len(reqs) // 2]
            mesh, rho, lam, mu, dt = serving.request_problem(r)
            d = bf.GpuDomain(mesh, rho, lam, mu, precision=prec, device=local)
            d.set_source(r.source, r.force, r.f0, r.t0)
            d.set_receivers(r.receivers, r.nsteps)
            bf.LSRK(d).step(dt, r.nsteps, use_graph=True)
            checks.append({"rate": rate, "request": r.id,
                           "alone_equals_in_mix": bool(np.array_equal(d.seismograms(),
                                                                      r.seismograms))})
            d.free()
    launches = bf.launch_count() - n0
    worst = max(c.get("rel_l2_vs_fp64_oracle", 0.0) for c in checks)
    if rank == 0:
        top = max(runs, key=lambda s: s["dof_updates_per_s"])
        line = {
            "metric": "DOF-updates/s (serving; p50/p99 latency per rate)",
            "value": top["dof_updates_per_s"], "unit": "DOF-updates/s",
            "n_gpus": ws, "steps": sum(s["chunks"] for s in runs), "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 rhs / f64 state" if prec == bf.PRECISION_FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": "cfg4: Poisson request streams (seed 2), bricks 8^3-24^3, "
                                   "N in {3,5}, 50-400 LSRK steps, Ricker point force, "
                                   "16 receivers, 150 GB budget, continuous batching",
                       "requests_per_rate": args.requests, "chunk_steps": args.chunk,
                       "parallelism": f"replicas{ws}"},
            "serving": runs, "accuracy": {"max_rel_l2_vs_fp64_oracle": worst,
                                          "checks": checks},
            "roofline": None, "cpu_baseline": None, "e2e": None,
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    return 0


def run_next_rows(args):
    """The rows beside the hot path, measured on the cfg1 mesh family:
    boundary faces (a bounded brick), glue between orders (two glued halves
    stepped in one batch, beside the same halves unglued), and element
    geometry computed on the device from quadrant data (domain set-up
    time).  Device-timed with CUDA events; set-up on the host clock."""
    import time
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    import bfam_b200 as bf
    from bfam_b200 import configs

    n, N, steps = args.n, 5, args.steps
    stream = torch.cuda.Stream(device=local)

    def time_domain(dom, dt):
        dom.set_stream(stream.cuda_stream)
        ts = bf.LSRK(dom)
        ts.step(dt, max(3, args.warmup), use_graph=True)
        dom.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ts.step(dt, steps, use_graph=True)
        e1.record(stream)
        e1.synchronize()
        ts.free()
        return e0.elapsed_time(e1) / 1e3

    def time_batch(b, dts):
        b.set_stream(stream.cuda_stream)
        b.step(dts, max(3, args.warmup))
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step(dts, steps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    out = {}
    with ClockSampler(local) as clk:
        # periodic and bounded cfg1-family bricks
        res = {}
        for name, periodic in (("periodic", (True,) * 3), ("bounded", (False,) * 3)):
            m = bf.Mesh(3, N, (n,) * 3, refine_prob=0.3, seed=0, periodic=periodic)
            rho, lam, mu = bf.material_random(m.K, 0)
            q0 = m.gaussian_pulse(bf.lgl_operators(N)[0], (0.5, 0.5, 0.5), 0.05)
            dt = configs.stable_dt(m, rho, lam, mu, 0.5)
            bc = (bf.BC_ABSORBING,) * 5 + (bf.BC_FREE_SURFACE,)
            d = bf.GpuDomain(m, rho, lam, mu, bc=bc, device=local)
            d.set_fields(q0)
            t = time_domain(d, dt)
            res[name] = {"dof_updates_per_s": m.ndof * 5 * steps / t, "elements": m.K,
                         "boundary_faces": int(m.Kb)}
            d.free()
        out["boundary"] = res
        # glued halves (orders 3 | 5 and 5 | 5) against the same halves unglued
        rng = np.random.default_rng(0)
        glue = {}
        for Na, Nb in ((5, 5), (3, 5)):
            row = {}
            # the same refinement for both runs; none next to the glued sides
            flag_sets = []
            for _ in range(2):
                flags = (rng.random((n, n, n // 2)) < 0.3).astype(np.uint8)
                flags[..., 0] = 0
                flags[..., -1] = 0
                flag_sets.append(flags)
            for glued in (True, False):
                meshes = []
                for Nn, flags in zip((Na, Nb), flag_sets):
                    per = (False, True, True) if glued else (True, True, True)
                    meshes.append(bf.Mesh(3, Nn, (n // 2, n, n), L=(0.5, 1.0, 1.0),
                                          refine_flags=flags.reshape(-1), periodic=per))
                doms, dts, dofs = [], [], 0
                for m in meshes:
                    rho, lam, mu = bf.material_random(m.K, 1)
                    bc = (bf.BC_GLUED, bf.BC_GLUED) + (bf.BC_FREE_SURFACE,) * 4
                    d = bf.GpuDomain(m, rho, lam, mu, bc=bc, device=local)
                    d.set_fields(m.gaussian_pulse(bf.lgl_operators(m.N)[0],
                                                  (0.25, 0.5, 0.5), 0.05))
                    doms.append(d)
                    dts.append(configs.stable_dt(m, rho, lam, mu, 0.5))
                    dofs += m.ndof
                b = bf.Batch(doms)
                if glued:
                    g = bf.PGlue(doms[0], doms[1], *bf.glued_x_pairs(*meshes))
                    b.add_pglue(g)
                dt = min(dts)
                t = time_batch(b, [dt, dt])
                row["glued" if glued else "unglued"] = {
                    "dof_updates_per_s": dofs * 5 * steps / t,
                    "launches_per_step": b.launches_per_step()}
                b.free()
                for d in doms:
                    d.free()
            glue[f"N{Na}|N{Nb}"] = row
        out["glue"] = glue
        # domain set-up: host geometry against geometry on the device
        m = bf.Mesh(3, N, (n,) * 3, refine_prob=0.3, seed=0)
        rho, lam, mu = bf.material_random(m.K, 0)
        geo = {}
        for mode in ("host", "device"):
            best = None
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                d = bf.GpuDomain(m, rho, lam, mu, geometry=mode, device=local)
                d.sync()
                t = time.perf_counter() - t0
                best = t if best is None else min(best, t)
                d.free()
            geo[mode] = {"create_s": best}
        geo["upload_bytes_per_element"] = {"host": 48, "device": 20}
        out["geometry"] = geo
    if rank == 0:
        line = {"metric": "DOF-updates/s", "value": out["boundary"]["bounded"]["dof_updates_per_s"],
                "unit": "DOF-updates/s", "n_gpus": ws, "steps": steps,
                "warmup": max(3, args.warmup), "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"rows beside the hot path on {n}^3 N={N} p=0.3 bricks: "
                                       "bounded brick, glued halves, device geometry"},
                **out, "roofline": None, "cpu_baseline": None, "e2e": None,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "cfg3":
        return run_batched(args)
    if args.config == "cfg2" and args.precision is None:
        return run_precision(args)
    if args.config == "cfg4":
        return run_serving(args)
    if args.config == "next":
        return run_next_rows(args)
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    import bfam_b200 as bf

    p = build_problem(args.config, args.n)
    prec = bf.PRECISION_FP32 if args.precision == "fp32" else bf.PRECISION_FP64
    dom = bf.GpuDomain(p.mesh, p.rho, p.lam, p.mu, precision=prec, device=local)
    stream = torch.cuda.Stream(device=local)
    dom.set_stream(stream.cuda_stream)
    dom.set_fields(p.q0)
    ts = bf.LSRK(dom)
    use_graph = bool(args.graph)
    for _ in range(max(3, args.warmup)):
        ts.step(p.dt, 1, use_graph=use_graph)
    dom.sync()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    n0 = bf.launch_count()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        ts.step(p.dt, args.steps, use_graph=use_graph)
        ev1.record(stream)
        ev1.synchronize()
    launches = bf.launch_count() - n0
    dom.sync()
    ms = ev0.elapsed_time(ev1)
    t_local = ms / 1e3
    t_max = max_over_ranks(t_local, local)
    if ws > 1:
        torch.distributed.barrier()
        torch.cuda.synchronize()
    ns = 5
    dof_updates = p.ndof * ns * args.steps
    value = replica_value(dof_updates, t_max, ws)

    # roofline of the dominant (only) kernel, the fused stage kernel, per
    # LSRK stage: one launch per refinement level (level 0, then the
    # elements with coarse-side hanging faces); the per-launch average gives
    # the same ratio
    levels = dom.launch_levels()
    per_stage_s = t_local / (ns * args.steps)
    alg_bytes_per_stage = p.ndof * ALG_BYTES_PER_DOF_UPDATE[ns]
    achieved = alg_bytes_per_stage / per_stage_s / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic(f"dg_stage_kernel_{p.name}") if p.mesh.dim == 3 else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"of {peak_kind}",
                "traffic": traffic,
                "kernel": "dg_stage_kernel (fused volume+face+mortar+LSRK update)",
                "per": f"LSRK stage = {levels} launch(es), one per refinement level",
                "alg_bytes_per_stage": alg_bytes_per_stage,
                "launches_per_stage": levels}

    # e2e: one full solve through the C-ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        host = torch.empty((dom.nfields, dom.field_length), dtype=torch.float64,
                           pin_memory=True)
        host_np = host.numpy()
        host_np[...] = p.q0
        out = torch.empty_like(host, pin_memory=True).numpy()
        tsolve = bf.LSRK(dom)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        dom.set_fields(host_np)
        ev[1].record(stream)
        tsolve.step(p.dt, p.nsteps, use_graph=use_graph)
        ev[2].record(stream)
        dom.get_fields(out)
        ev[3].record(stream)
        ev[3].synchronize()
        el = ev[0].elapsed_time(ev[3]) / 1e3
        phases = {k: ev[i].elapsed_time(ev[i + 1]) / 1e3
                  for i, k in enumerate(("upload_s", "steps_s", "download_s"))}
        el = max_over_ranks(el, local)
        nbytes = host_np.nbytes
        e2e = {"value": p.ndof * ns * p.nsteps * ws / el, "unit": "DOF-updates/s",
               "phases": phases,
               "steps_only_value": p.ndof * ns * p.nsteps / phases["steps_s"],
               "h2d_bytes_per_step": nbytes / p.nsteps,
               "d2h_bytes_per_step": nbytes / p.nsteps,
               "h2d_bytes_per_solve": nbytes, "d2h_bytes_per_solve": nbytes,
               "step": f"one LSRK step; the timed unit is one solve (upload the state, "
                       f"{p.nsteps} steps, download the state), so the copies are "
                       "counted per solve and per step amortised over it",
               "seconds": el}
        tsolve.free()

    # per-launch-level observability (event pair per launch, eager steps,
    # outside the timed region)
    dom.profile(True)
    ts.step(p.dt, 2, use_graph=False)
    per_level = dom.kernel_stats()
    dom.profile(False)
    for st in per_level:
        st["frac_of_peak"] = st["gbs"] / peak if peak else None

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(p)

    if rank == 0:
        line = {
            "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 rhs / f64 state" if prec == bf.PRECISION_FP32 else "f64",
            "data": "synthetic",
            "config": dict(workload_desc(p), parallelism=f"replicas{ws}",
                           cuda_graph=use_graph),
            "roofline": roofline, "per_launch_level": per_level,
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ts.free()
    dom.free()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
