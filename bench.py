#!/usr/bin/env python
"""Benchmark of the SharpClaw WENO step on B200 (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): 1-D Euler,
gamma = 1.4, Shu-Osher shock/entropy-wave data on [-5,5] with extrapolation
bc, mx = 2^20 cells, Roe solver with Harten-Hyman entropy fix
(apps/euler/shockentropy/rp1eu.f), characteristic-wise WENO5 with Roe
eigenvectors, tfluct_solver = 0 (swap + second Riemann solve), SSPRK(10,4),
cfl_desired 2.45 / cfl_max 2.5, variable dt.  Synthetic data of exactly that
recipe (no dataset is involved).

One benchmark step = one sharpclaw() call advancing the grid by 50 time
steps (500 fused stage launches + 51 controller launches), i.e.
2^20 * 50 * 10 cell-stage updates.

  value    device-resident throughput of the headline form (FP32
           reconstruction/Riemann on FP64 state, `--precision mixed`),
           CUDA events on the library stream, L2 flushed between steps
  fp64     the plain FP64 path on the same workload, same timing
  e2e      the public C ABI with host buffers: H2D of q from pinned memory,
           sharpclaw(), D2H of q, every step, host wall clock
  roofline the fused stage kernel against the measured HBM copy bandwidth
  cpu_baseline  the C oracle (a restatement of the reference Fortran, which
           cannot be compiled here: no Fortran compiler) on a bounded sample

`--impl reference` times that CPU restatement alone, on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-stage updates/s on 1 B200, FP32+batched vs plain FP64 at stated L1 err; %HBM"
UNIT = "cell-stage/s"
MX = 1 << 20
NSTEP = 50          # time steps per benchmark step
NSTAGES = 10        # SSPRK(10,4)
CFL_MAX, CFL_DESIRED = 2.5, 2.45
DT0 = 4.5e-6        # below 2.45*dx/max(|u|+c) of the Shu-Osher data: no rejected first step
GAMMA = 1.4
WORKLOAD = ("1-D Euler Shu-Osher, mx=2^20, Roe+entropy fix, char-wise WENO5, tfluct_solver=0, "
            "SSPRK(10,4), cfl 2.45/2.5, variable dt, extrapolation bc")


def shu_osher(mx):
    import numpy as np
    xlower, xupper = -5.0, 5.0
    dx = (xupper - xlower) / mx
    xc = xlower + (np.arange(1, mx + 1) - 0.5) * dx
    g1 = GAMMA - 1.0
    rhol, ul, pl = 3.857143, 2.629369, 10.333333
    q = np.zeros((3, mx + 6))
    left = xc < -4.0
    q[0, 3:-3] = np.where(left, rhol, 1.0 + 0.2 * np.sin(5.0 * xc))
    q[1, 3:-3] = np.where(left, rhol * ul, 0.0)
    q[2, 3:-3] = np.where(left, pl / g1 + 0.5 * rhol * ul ** 2, 1.0 / g1)
    return q, dx


def config(extra=None):
    c = {"workload": WORKLOAD, "cells": MX, "time_steps_per_step": NSTEP, "stages_per_time_step": NSTAGES,
         "l2": "flushed (256 MiB write) between timed steps",
         "parallelism": "replicas (one independent grid per GPU)"}
    if extra:
        c.update(extra)
    return c


# --------------------------------------------------------------------------
# CPU restatement (oracle) timing: used for cpu_baseline and --impl reference
# --------------------------------------------------------------------------
def _oracle_one(args):
    mx, nsteps = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    q, dx = shu_osher(mx)
    p = O.make_params(mx=mx, meqn=3, mwaves=3, dx=dx, xlower=-5.0, rp=O.RP_EULER, gamma=GAMMA,
                      mthbc=(1, 1), char_decomp=2, tfluct_solver=0)
    t0 = time.perf_counter()
    qq, res = O.sharpclaw(p, q, None, tstart=0.0, tend=1e30, dt_initial=DT0, cfl_max=CFL_MAX,
                          cfl_desired=CFL_DESIRED, max_steps=nsteps, time_integrator=4)
    dt = time.perf_counter() - t0
    return mx * NSTAGES * res.steps_taken, dt


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# --------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# --------------------------------------------------------------------------
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        import statistics
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 3 + k and s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------------------
def run_reference(args, rank, world):
    """--impl reference: the CPU restatement on all host cores (rank 0 only)."""
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = cpu_cores()
    sample_mx = MX                      # the headline grid itself
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_oracle_one, [(1024, 1)] * cores)  # import + warm the workers
        for _ in range(args.warmup):
            pool.map(_oracle_one, [(sample_mx, 1)] * cores)
        rates, walls = [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            out = pool.map(_oracle_one, [(sample_mx, 1)] * cores)
            wall = time.perf_counter() - t0
            walls.append(wall)
            rates.append(sum(n for n, _ in out) / wall)
    value = sum(rates) / len(rates)
    ms = 1000.0 * sum(walls) / len(walls)
    sample = (f"{cores} independent processes on {cores} host cores ({cpu_model()}), each one "
              f"SSPRK(10,4) time step of the headline Shu-Osher grid, mx=2^20 (C restatement of the "
              f"reference, gcc -O2, no FMA)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config({"sample_mx": sample_mx, "host_cpu": cpu_model()}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample, "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(x, world, device):
    """Largest x over all ranks (an all-reduce, so every rank receives it)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world, device):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units, seconds, world, device):
    """Whole-job throughput: the units every rank processed, summed, over the
    slowest rank's time.  Returns (rate, slowest time).  Every rank must call
    it, in the same order as the other collectives."""
    tmax = max_over_ranks(seconds, world, device)
    return sum_over_ranks(units, world, device) / tmax, tmax


def oracle_params(ps):
    """The oracle's parameter struct for the same run as ClawParams ps."""
    from oracle import oracle as O
    return O.make_params(ndim=ps.ndim, mx=ps.mx, my=ps.my, meqn=ps.meqn, mwaves=ps.mwaves, mbc=ps.mbc,
                         maux=ps.maux, mcapa=ps.mcapa, char_decomp=ps.char_decomp, tfluct_solver=ps.tfluct_solver,
                         mthbc=tuple(ps.mthbc), dx=ps.dx, dy=ps.dy, xlower=ps.xlower, ylower=ps.ylower, rp=ps.rp,
                         efix=ps.efix, u=ps.u, gamma=ps.gamma, grav=ps.grav, lim_type=ps.lim_type,
                         mthlim=tuple(ps.mthlim), src_term=ps.src_term, rho=ps.rho, bulk=ps.bulk)


def shu_osher_params(S, mx, dx):
    return S.ClawParams(rp=S.RP_EULER, mx=mx, dx=dx, xlower=-5.0, gamma=GAMMA, mthbc=(1, 1),
                        char_decomp=2, tfluct_solver=0, time_integrator=4)


def workloads():
    """Benchmark workloads c1..c5 (1-D advection 1000 cells, 1-D Euler 2^20,
    2-D shallow water 4096^2, batched Riemann problems, 2-D acoustics 1024^2
    with its adjoint).  Each returns the solver
    parameters, initial data, aux, run settings and the bytes one cell-stage
    must move (k_I * meqn * 8 + maux * 8, double state)."""
    import numpy as np
    import sharpclaw_b200 as S

    def c2():
        q, dx = shu_osher(MX)
        return dict(params=shu_osher_params(S, MX, dx), q=q, aux=None, dt0=DT0, cfl=(CFL_MAX, CFL_DESIRED),
                    dt_variable=1, tend=1e30, nstep=NSTEP, cells=MX, stages=10, bytes_cell_stage=2.3 * 3 * 8,
                    desc=WORKLOAD, traffic_key="k_stage1d_euler_charwise_mixed", oracle_steps=2)

    def c1():
        mx = 1000
        dx = 1.0 / mx
        rng = np.random.default_rng(1)
        xc = (np.arange(mx) + 0.5) * dx
        q0 = np.exp(-200.0 * (xc - 0.3) ** 2) + ((xc > 0.6) & (xc < 0.8))
        for _ in range(4):
            k = rng.integers(1, 9)
            q0 = q0 + rng.uniform(0, 0.1) * np.sin(2 * np.pi * k * xc)
        q = np.zeros((1, mx + 6))
        q[0, 3:-3] = q0
        p = S.ClawParams(rp=S.RP_ADVECTION, mx=mx, dx=dx, u=1.0, mthbc=(2, 2), char_decomp=0,
                         tfluct_solver=1, time_integrator=3)
        return dict(params=p, q=q, aux=None, dt0=0.8 * dx, cfl=(0.85, 0.8), dt_variable=1, tend=1.0,
                    nstep=2000, cells=mx, stages=3, bytes_cell_stage=8.0 / 3.0 * 8,
                    desc="1-D advection a=1, periodic [0,1], mx=1000, WENO5 componentwise + Godunov rp, "
                         "tfluct, SSPRK3, cfl 0.8/0.85, full run to t=1 per step", traffic_key=None,
                    oracle_steps=20)

    def c3():
        n = 4096
        d = 5.0 / n
        xc = -2.5 + (np.arange(n) + 0.5) * d
        X, Y = np.meshgrid(xc, xc, indexing="xy")
        q = np.zeros((3, n + 6, n + 6))
        q[0, 3:-3, 3:-3] = np.where(X ** 2 + Y ** 2 < 0.25, 2.0, 1.0) + \
            1e-3 * np.random.default_rng(3).standard_normal((n, n))
        p = S.ClawParams(rp=S.RP_SW2D, mx=n, my=n, dx=d, dy=d, xlower=-2.5, ylower=-2.5, grav=1.0,
                         mthbc=(2, 2, 2, 2), char_decomp=2, tfluct_solver=1, time_integrator=3)
        return dict(params=p, q=q, aux=None, dt0=0.3 * d / 1.5, cfl=(0.5, 0.45), dt_variable=1, tend=1e30,
                    nstep=5, cells=n * n, stages=3, bytes_cell_stage=8.0 / 3.0 * 3 * 8,
                    desc="2-D shallow water g=1, radial dam break h=2 in r<0.5 else 1 + N(0,1e-3), "
                         "4096x4096 periodic on [-2.5,2.5]^2, Roe rpn2 + tfluct, char-wise WENO5, SSPRK3, "
                         "cfl 0.45/0.5", traffic_key="k_stage2d_sw_charwise_mixed", oracle_steps=1)

    def c5():
        n = 1024
        d = 1.0 / n
        rng = np.random.default_rng(5)
        ln = rng.normal(0, 0.3, (2, n, n))
        ker = np.exp(-0.5 * (np.arange(-12, 13) / 4.0) ** 2)
        ker /= ker.sum()
        for a in ln:                      # periodic Gaussian smoothing (sigma = 4 cells)
            for ax in (0, 1):
                a[...] = sum(w * np.roll(a, s, axis=ax) for s, w in zip(range(-12, 13), ker))
        rho, K = np.exp(ln[0]), np.exp(ln[1])
        inner = np.stack([np.sqrt(rho * K), np.sqrt(K / rho)])
        aux = np.ascontiguousarray(np.pad(inner, ((0, 0), (3, 3), (3, 3)), mode="wrap"))
        xc = (np.arange(-3, n + 3) + 0.5) * d
        X, Y = np.meshgrid(xc, xc, indexing="xy")
        q = np.zeros((3, n + 6, n + 6))
        for _ in range(4):
            cx, cy = rng.uniform(0.2, 0.8, 2)
            q[0] += np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * 0.03 ** 2))
        # smooth background: keeps every cell's WENO smoothness indicators far
        # above epsilon, where the adjoint (a derivative) is well conditioned
        q[0] += 0.05 * np.cos(2 * np.pi * X) * np.cos(2 * np.pi * Y)
        p = S.ClawParams(rp=S.RP_ACOUSTICS2D, mx=n, my=n, dx=d, dy=d, mthbc=(2, 2, 2, 2), char_decomp=0,
                         tfluct_solver=1, time_integrator=3)
        dt = 0.4 * d / float(aux[1].max())
        return dict(params=p, q=q, aux=aux, dt0=dt, cfl=(1e9, 0.5), dt_variable=0, tend=20 * dt,
                    nstep=20, cells=n * n, stages=3, bytes_cell_stage=8.0 / 3.0 * 3 * 8 + 2 * 8,
                    desc="2-D variable-coefficient acoustics 1024x1024 periodic, rho,K log-normal(0,0.3) "
                         "smoothed (periodic), p0 = 4 Gaussian bumps + 0.05 cos cos, WENO5 componentwise + "
                         "rpn2/tfluct, SSPRK3, fixed dt, 20 steps per step", traffic_key="k_stage2d_acoustics_mixed",
                    oracle_steps=2)

    return {"c2": c2, "c1": c1, "c3": c3, "c5": c5}


def run_gpu(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    import sharpclaw_b200 as S

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    W = workloads()[args.workload]()
    ps, q0, aux0 = W["params"], W["q"], W["aux"]
    cfl_max, cfl_des = W["cfl"]
    nstep = W["nstep"]
    cells = W["cells"] * nstep * W["stages"]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_steps(s):
        return s.time_steps(nstep, W["dt0"], cfl_max, cfl_des, tend=W["tend"], dt_variable=W["dt_variable"])

    def device_run(precision, clocks, totals=False):
        s = S.Solver(ps, precision)
        if totals:
            s.set_totals(True)
        if aux0 is not None:
            s.set_aux(aux0)
        s.set_q(q0)
        for _ in range(args.warmup):
            if W["tend"] < 1e29:
                s.set_q(q0)
            timed_steps(s)
        barrier()
        total_ms, taken, rejected = 0.0, 0, 0
        with clocks:
            for _ in range(args.steps):
                if W["tend"] < 1e29:          # runs to a final time restart from q0
                    s.set_q(q0)
                flush.zero_()
                torch.cuda.synchronize()
                ms, res = timed_steps(s)
                assert res["status"] == 0 and res["info"] in (0, 11), res
                total_ms += ms
                taken += res["steps_taken"] - res["rejected"]
                rejected += res["rejected"]
                run_record = s.last_run()
        barrier()
        s.timed_run_record = run_record
        return s, total_ms, res, taken, rejected

    clocks = Clocks(local_rank)
    s_mix, ms_mix, res_mix, taken_mix, rej_mix = device_run(args.precision, clocks)
    value, s_max = job_rate(W["cells"] * W["stages"] * taken_mix, ms_mix / 1000.0, world, dev)
    ms_mix = 1000.0 * s_max
    s_64, ms_64, res_64, taken_64, rej_64 = device_run("fp64", clocks)
    value64, s_max = job_rate(W["cells"] * W["stages"] * taken_64, ms_64 / 1000.0, world, dev)
    ms_64 = 1000.0 * s_max
    # the headline form with the FP64 conserved-total bookkeeping on (one
    # compensated-sum kernel per step); the drift is the largest change of
    # the totals over a timed run (boundary fluxes included: this grid has
    # extrapolation boundaries)
    s_tot, ms_tot, _, taken_tot, _ = device_run(args.precision, clocks, totals=True)
    value_tot, _ = job_rate(W["cells"] * W["stages"] * taken_tot, ms_tot / 1000.0, world, dev)
    T = s_tot.conserved_totals()
    totals = {"value": value_tot, "unit": UNIT, "overhead": value / value_tot - 1.0,
              "tot0": T["tot0"].tolist(), "tot": T["tot"].tolist(), "drift": T["drift"].tolist(),
              "note": "one FP64 compensated-sum kernel per time step; totals of the last timed run"}
    s_tot.close()

    # the fused stage kernels alone (roofline): the stage launches of one step
    peak, peak_kind = measured_peaks()
    traffic_per_cell = None
    if W["traffic_key"]:
        try:
            with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
                traffic_per_cell = json.load(f)[W["traffic_key"]]["dram_bytes_per_cell"]
        except Exception:
            traffic_per_cell = None
    counters = {}
    if W["traffic_key"]:
        try:
            with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
                counters = json.load(f)
        except Exception:
            counters = {}
    roof = {}
    for name, s in (("headline", s_mix), ("fp64", s_64)):
        st_ms, n_launch = s.time_stages(res_mix["dt_last"], 20)
        avg_ms = st_ms / n_launch
        bytes_per_launch = W["bytes_cell_stage"] * W["cells"]
        gbs = bytes_per_launch / (avg_ms / 1000.0) / 1e9
        roof[name] = {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                      "frac": gbs / peak,
                      "traffic": (traffic_per_cell * W["cells"]) if traffic_per_cell else None,
                      "avg_launch_us": avg_ms * 1000.0, "algorithmic_bytes_per_launch": bytes_per_launch,
                      "peak_source": peak_kind}
        # the issue-slot ceiling of the same kernel: warp instructions per
        # cell-stage (ncu capture of the kernel, profiles/) at the measured
        # launch rate, against 4 schedulers x SMs x the SM clock under load
        key = W["traffic_key"] and W["traffic_key"].replace("_mixed", "_" + ("fp64" if name == "fp64" else args.precision))
        wi = counters.get(key, {}).get("warp_inst_per_cell") if key else None
        roof[name]["compute_key"] = key
        roof[name]["warp_inst_per_cell_stage"] = wi
        # this form's own DRAM bytes per cell when its kernel was captured
        tpc = counters.get(key, {}).get("dram_bytes_per_cell") if key else None
        if tpc:
            roof[name]["traffic"] = tpc * W["cells"]

    # end to end through the public API with host buffers
    qh = torch.from_numpy(q0.copy()).pin_memory()
    qout = torch.empty_like(qh).pin_memory()
    qh_np, qout_np = qh.numpy(), qout.numpy()
    s_e2e = s_mix

    def e2e_step():
        s_e2e.set_q(qh_np)
        r = s_e2e.sharpclaw(0.0, W["tend"], W["dt0"], cfl_max, cfl_des, max_steps=nstep,
                            dt_variable=W["dt_variable"])
        _get_q_into(s_e2e, qout_np)
        return r

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e2e_taken = 0
    with clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = e2e_step()
            e2e_taken += r["steps_taken"] - r["rejected"]
        barrier()
        e2e_local = time.perf_counter() - t0
    e2e, e2e_s = job_rate(W["cells"] * W["stages"] * e2e_taken, e2e_local, world, dev)
    nbytes = q0.nbytes

    # accuracy against the oracle (the C restatement of the reference, run
    # here on one host core) over a short fixed-dt window of the same grid,
    # and against the GPU's FP64_STRICT form (bit for bit the oracle, by the
    # GPU tests) over a longer one
    acc = {}
    if rank == 0:
        from oracle import oracle as O

        def inner(q):
            return q[:, 3:-3] if ps.ndim == 1 else q[:, 3:-3, 3:-3]

        def rel_l1(a, b):
            return max(float(np.abs(a[m] - b[m]).sum() / max(np.abs(b[m]).sum(), 1e-300)) for m in range(a.shape[0]))

        def rel_linf(a, b):
            return float(np.abs(a - b).max() / np.abs(b).max())

        def gpu_run(name, nsteps):
            with S.Solver(ps, name) as s:
                if aux0 is not None:
                    s.set_aux(aux0)
                s.set_q(q0)
                s.sharpclaw(0.0, nsteps * dt, dt, 1e9, 0.5, dt_variable=0)
                return inner(s.get_q())

        dt = W["dt0"]
        n_or = W["oracle_steps"]
        t0 = time.perf_counter()
        qo, _ = O.sharpclaw(oracle_params(ps), q0, aux0, tstart=0.0, tend=n_or * dt, dt_initial=dt, cfl_max=1e9,
                            cfl_desired=0.5, dt_variable=0, time_integrator=ps.time_integrator)
        oracle_s = time.perf_counter() - t0
        b = inner(qo)
        vs_oracle = {"steps": n_or, "dt": dt, "oracle_seconds": oracle_s}
        for name in (args.precision, "fp64", "fp64_strict"):
            a = gpu_run(name, n_or)
            vs_oracle[name] = {"rel_l1": rel_l1(a, b), "rel_linf": rel_linf(a, b),
                               "bitwise_equal": bool(np.array_equal(a, b))}
        outs = {name: gpu_run(name, 20) for name in ("fp64_strict", args.precision, "fp64")}
        a, b = outs[args.precision], outs["fp64_strict"]
        acc = {"vs_oracle": vs_oracle,
               "rel_l1_vs_fp64_strict": rel_l1(a, b), "rel_linf_vs_fp64_strict": rel_linf(a, b),
               "fp64_rel_linf_vs_fp64_strict": rel_linf(outs["fp64"], b), "steps": 20, "dt": dt}

    # CPU baseline: the oracle on a bounded sample, one core (C2 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and args.workload == "c2":
        n, t = _oracle_one((MX, 1))
        cpu = {"value": n / t, "unit": UNIT, "cores": 1, "kind": "port", "cpu_model": cpu_model(),
               "sample": "the headline grid, mx=2^20 Shu-Osher, 1 SSPRK(10,4) time step, C restatement of the "
                         "reference (gcc -O2, no FMA), single thread"}

    # the batched workload (2048 Riemann problems), a short window, in the
    # same process: FP32 batch against plain FP64 run one grid at a time
    batched = None
    if args.workload == "c2" and not args.no_batched:
        batched, bout = batch_measure(args, world, dev, C4_BLOCK_TEND, 3, 1, clocks, flush, e2e=False,
                                      one_at_a_time=24)
        for v in bout.values():
            v["batch"].close()

    adj = None
    if args.workload == "c5" and rank == 0:
        adj = c5_adjoint(S, ps, q0, aux0, W["dt0"])

    # the other single-grid configurations, a few timed steps each in the
    # same process and the same way as the headline (device-resident state,
    # L2 flushed between steps, CUDA events), headline form and plain FP64
    others = None
    if args.workload == "c2" and not args.no_batched:
        others = {}
        for wname in ("c1", "c3", "c5"):
            Wo = workloads()[wname]()
            entry = {"workload": Wo["desc"], "cells": Wo["cells"], "time_steps_per_step": Wo["nstep"]}
            for prec in (args.precision, "fp64"):
                key = "fp64" if prec == "fp64" else "headline"
                try:
                    rate, ms, mode = quick_config(S, Wo, prec, 3, 2, flush, world, dev, barrier)
                except Exception as e:   # never lose the headline line to this block
                    entry[key] = {"error": f"{type(e).__name__}: {e}"}
                    continue
                entry[key] = {"value": rate, "unit": UNIT, "precision": prec, "ms_per_step": ms,
                              "time_loop": "cluster-resident launch" if mode == S.RUN_RESIDENT else "CUDA graphs"}
            others[wname] = entry

    # kernels the library launched in one timed sharpclaw loop (graph nodes
    # counted one by one; one launch per 4096 steps for a cluster-resident run)
    run_mode, run_launches = s_mix.timed_run_record
    launches = run_launches * args.steps
    ck = clocks.summary()
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    for name, r in roof.items():
        wi = r.pop("warp_inst_per_cell_stage")
        key = r.pop("compute_key")
        if wi and ck.get("sm_mhz"):
            rate = W["cells"] / (r["avg_launch_us"] * 1e-6)     # cell-stages per second of the kernel
            ach = wi * rate
            pk = nsm * 4 * ck["sm_mhz"] * 1e6
            r["compute"] = {"bound": "issue", "unit": "warp-instructions/s", "achieved": ach, "peak": pk,
                            "frac": ach / pk, "warp_inst_per_cell_stage": wi, "counters": key,
                            "peak_is": f"{nsm} SMs x 4 schedulers x median SM clock under load"}
    if rank == 0:
        cfg = {"workload": W["desc"], "cells": W["cells"], "time_steps_per_step": nstep,
               "stages_per_time_step": W["stages"], "precision": args.precision,
               "l2": "flushed (256 MiB write) between timed steps",
               "parallelism": "replicas (one independent grid per GPU)",
               "time_loop": "cluster-resident launch" if run_mode == S.RUN_RESIDENT else "CUDA graphs"}
        if ps.ndim == 2:
            cfg["tiles"] = {"headline": s_mix.tiles(), "fp64": s_64.tiles()}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_mix / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": {"mixed": "f32 (f64 state/accumulation)", "fp32": "f32", "fp64": "f64",
                          "fp64_strict": "f64"}[args.precision],
                "data": "synthetic", "config": cfg,
                "roofline": roof["headline"],
                "fp64": {"value": value64, "unit": UNIT, "ms_per_step": ms_64 / args.steps,
                         "roofline": roof["fp64"], "speedup_of_headline": value / value64},
                "rejected_steps": rej_mix,
                "totals": totals,
                "accuracy": acc,
                "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                        "ms_per_step": 1000.0 * e2e_s / args.steps},
                "gpu_launches": launches,
                "clocks": ck}
        if adj is not None:
            line["adjoint"] = adj
        if batched is not None:
            line["batched"] = batched
        if others is not None:
            line["other_configs"] = others
        print(json.dumps(line), flush=True)
    s_mix.close()
    s_64.close()
    return 0


def quick_config(S, W, precision, steps, warmup, flush, world, dev, barrier):
    """Cell-stage rate of workload W in one arithmetic form: `warmup` untimed
    then `steps` timed runs of W's step (time_steps on the device-resident
    state, CUDA events inside the library), L2 flushed before each; the
    slowest rank's time.  Returns (rate, ms per step, run mode)."""
    import torch
    ps, q0, aux0 = W["params"], W["q"], W["aux"]
    cfl_max, cfl_des = W["cfl"]
    s = S.Solver(ps, precision)
    try:
        if aux0 is not None:
            s.set_aux(aux0)
        s.set_q(q0)

        def one():
            if W["tend"] < 1e29:
                s.set_q(q0)
            flush.zero_()
            torch.cuda.synchronize()
            return s.time_steps(W["nstep"], W["dt0"], cfl_max, cfl_des, tend=W["tend"],
                                dt_variable=W["dt_variable"])

        for _ in range(warmup):
            one()
        barrier()
        total_ms, taken = 0.0, 0
        for _ in range(steps):
            ms, res = one()
            assert res["status"] == 0 and res["info"] in (0, 11), res
            total_ms += ms
            taken += res["steps_taken"] - res["rejected"]
        barrier()
        rate, s_max = job_rate(W["cells"] * W["stages"] * taken, total_ms / 1000.0, world, dev)
        return rate, 1000.0 * s_max / steps, s.last_run()[0]
    finally:
        s.close()


def c5_adjoint(S, ps, q0, aux0, dt, nsteps=200, ckpt=20):
    """Gradient of J = 1/2||p(T) - p_obs||^2 with respect to the initial
    pressure through 200 SSPRK(3,3) steps (checkpoint every 20, hand-written
    FP64 adjoint), timed; checked against central differences along a smooth
    direction and against the gradient linearised at mixed-precision states."""
    import numpy as np
    import torch
    from sharpclaw_b200 import adjoint as A
    rng = np.random.default_rng(55)
    n = ps.mx
    inner = q0[0, 3:-3, 3:-3]
    p_obs = torch.from_numpy(np.ascontiguousarray(0.9 * inner)).cuda()
    p0 = torch.from_numpy(np.ascontiguousarray(inner)).cuda()
    out = {}
    grads = {}
    for precision in ("fp64", "mixed"):
        with S.Solver(ps, precision) as s:
            s.set_aux(aux0)
            x = p0.clone().requires_grad_(True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            J = A.wave_misfit(x, s, dt, nsteps, p_obs, checkpoint_every=ckpt)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            (g,) = torch.autograd.grad(J, x)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            grads[precision] = g
            out[precision] = {"forward_s": t1 - t0, "backward_s": t2 - t1, "J": float(J.detach())}
            if precision == "fp64":
                xc = (np.arange(n) + 0.5) / n
                X, Y = np.meshgrid(xc, xc, indexing="xy")
                dvec = torch.from_numpy(np.sin(2 * np.pi * (X + 2 * Y)) * np.cos(4 * np.pi * X)).cuda()
                h = 1e-6
                Jp = A.wave_misfit(p0 + h * dvec, s, dt, nsteps, p_obs)
                Jm = A.wave_misfit(p0 - h * dvec, s, dt, nsteps, p_obs)
                fd = float((Jp - Jm) / (2 * h))
                ad = float((g * dvec).sum())
                out["fd_check"] = {"direction": "sin(2pi(x+2y)) cos(4pi x)", "h": h, "fd": fd, "adjoint": ad,
                                   "rel_err": abs(fd - ad) / abs(fd)}
    g64, gm = grads["fp64"], grads["mixed"]
    out["mixed_vs_fp64_gradient_rel_l2"] = float(torch.linalg.norm(gm - g64) / torch.linalg.norm(g64))
    out["steps"], out["checkpoint_every"], out["grid"] = nsteps, ckpt, f"{n}x{n}"
    return out


C4_TEND = 0.005     # bounded window of the batched workload (the full run ends at t = 0.2)


def c4_instances(n=2048, seed=4):
    """2048 1-D Euler Riemann problems on [0,1], jump at x = 0.5,
    mx ~ round(exp(U[ln 256, ln 65536])), left/right rho, p ~ U[0.1,1],
    u ~ U[-1,1], gamma = 1.4, extrapolation bc (seeded)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    mx = np.rint(np.exp(rng.uniform(np.log(256), np.log(65536), n))).astype(np.int32)
    rho = rng.uniform(0.1, 1.0, (n, 2))
    u = rng.uniform(-1.0, 1.0, (n, 2))
    p = rng.uniform(0.1, 1.0, (n, 2))
    qs, dt0 = [], []
    for k in range(n):
        m = int(mx[k])
        xc = (np.arange(m) + 0.5) / m
        left = xc < 0.5
        r = np.where(left, rho[k, 0], rho[k, 1])
        v = np.where(left, u[k, 0], u[k, 1])
        pr = np.where(left, p[k, 0], p[k, 1])
        q = np.zeros((3, m + 6))
        q[0, 3:-3], q[1, 3:-3], q[2, 3:-3] = r, r * v, pr / 0.4 + 0.5 * r * v * v
        qs.append(q)
        smax = float(np.max(np.abs(u[k]) + np.sqrt(1.4 * p[k] / rho[k])))
        dt0.append(0.5 / m / smax)
    return mx, 1.0 / mx.astype(np.float64), qs, np.array(dt0)


C4_BLOCK_TEND = 0.001   # window of the batched block inside the default (headline) run


def batch_measure(args, world, dev, tend, steps, warmup, clocks, flush, e2e=True, one_at_a_time=48):
    """The batched workload (2048 Riemann problems) over t in [0, tend]: the
    batched solver in the FP32 form (the headline of this workload), the mixed
    form, FP64 and FP64_STRICT (the oracle's operation order: bit for bit the
    oracle's sharpclaw() per instance, by the GPU tests), plus FP64 run one
    grid at a time on a seeded sample.  Device time with CUDA events, L2
    flushed between timed runs.  Returns a dict of rates, accuracy (per
    instance, largest relative L1 over the components against the FP64_STRICT
    batch) and the batches (open; the caller closes them)."""
    import numpy as np
    import torch
    import sharpclaw_b200 as S
    mx, dx, qs, dt0 = c4_instances()
    ps = S.ClawParams(rp=S.RP_EULER, mx=10, dx=0.1, mthbc=(1, 1), char_decomp=0, tfluct_solver=0,
                      time_integrator=3, gamma=GAMMA)
    cfl_max, cfl_des = 0.9, 0.8

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def cell_stages(res):
        return sum(int(mx[k]) * 3 * (r["steps_taken"] - r["rejected"]) for k, r in enumerate(res))

    out = {}
    for precision in ("fp32", "mixed", "fp64", "fp64_strict"):
        b = S.Batch(ps, mx, dx, precision=precision)
        for _ in range(warmup):
            b.set_q(qs)
            b.sharpclaw(0.0, tend, dt0, cfl_max, cfl_des)
        barrier()
        tot_ms, tot_cells, tot_launch = 0.0, 0, 0
        with clocks:
            for _ in range(steps):
                b.set_q(qs)
                flush.zero_()
                torch.cuda.synchronize()
                res, ms = b.sharpclaw(0.0, tend, dt0, cfl_max, cfl_des)
                tot_ms += ms
                tot_cells += cell_stages(res)
                tot_launch += b.launches()
        barrier()
        # instances the scheme cannot advance (a non-finite state: WENO5 is not
        # positivity preserving near vacuum) are flagged, not trapped
        failed = {int(k): r["info"] for k, r in enumerate(res) if r["info"] != 0}
        rate, s_max = job_rate(tot_cells, tot_ms / 1000.0, world, dev)
        out[precision] = dict(batch=b, ms=1000.0 * s_max, cells=tot_cells, rate=rate, res=res, tune=b.tuning(),
                              failed=failed, launches=tot_launch)

    # plain FP64 path with the instances run one at a time (a seeded sample)
    rng = np.random.default_rng(44)
    sample = rng.choice(len(mx), one_at_a_time, replace=False)
    one_ms, one_cells = 0.0, 0
    for k in sample:
        p1 = S.ClawParams(rp=S.RP_EULER, mx=int(mx[k]), dx=float(dx[k]), mthbc=(1, 1), char_decomp=0,
                          tfluct_solver=0, time_integrator=3, gamma=GAMMA)
        with S.Solver(p1, "fp64") as s:
            s.set_q(qs[k])
            ms, r = s.time_steps(200000, float(dt0[k]), cfl_max, cfl_des, tend=tend)
            one_ms += ms
            one_cells += int(mx[k]) * 3 * (r["steps_taken"] - r["rejected"])
    one_rate, _ = job_rate(one_cells, one_ms / 1000.0, world, dev)

    ref = out["fp64_strict"]["batch"].get_q()

    def accuracy(form):
        got = out[form]["batch"].get_q()
        bad = set(out[form]["failed"]) | set(out["fp64_strict"]["failed"])
        e = np.asarray([max(float(np.abs(g[m, 3:-3] - f[m, 3:-3]).sum() / np.abs(f[m, 3:-3]).sum())
                            for m in range(3)) for k, (g, f) in enumerate(zip(got, ref)) if k not in bad])
        return {"rel_l1_vs_fp64_strict_max_over_instances": float(e.max()),
                "rel_l1_vs_fp64_strict_median": float(np.median(e)),
                "instances_compared": int(e.size), "instances_above_1e-5": int((e > 1e-5).sum()),
                "nonfinite_instances": len(out[form]["failed"])}

    e2e_rate = None
    nbytes = 0
    if e2e:
        import ctypes
        from sharpclaw_b200 import _capi as C
        bh = out["fp32"]["batch"]
        flat = torch.from_numpy(bh.pack(qs)).pin_memory()
        flat_np = flat.numpy()
        outbuf = torch.empty_like(flat).pin_memory().numpy()
        nbytes = int(flat_np.nbytes)
        barrier()
        with clocks:
            t0 = time.perf_counter()
            e2e_cells = 0
            for _ in range(steps):
                C.check(C.lib().scl_batch_set_q(bh._h, flat_np.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                        "set_q")
                res, _ = bh.sharpclaw(0.0, tend, dt0, cfl_max, cfl_des)
                C.check(C.lib().scl_batch_get_q(bh._h, outbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                        "get_q")
                e2e_cells += cell_stages(res)
            barrier()
            e2e_rate, e2e_s = job_rate(e2e_cells, time.perf_counter() - t0, world, dev)
    r32, r64, r64s = out["fp32"]["rate"], out["fp64"]["rate"], out["fp64_strict"]["rate"]
    summary = {
        "workload": ("2048 batched 1-D Euler Riemann problems, mx~log-uniform[256,65536] (seed 4), rho,p U[0.1,1], "
                     f"u U[-1,1], WENO5 componentwise + Roe/efix, SSPRK3, cfl 0.8/0.9, window t in [0,{tend}]"),
        "cells_total": int(mx.sum()), "instances": len(mx), "window": tend, "timed_runs": steps,
        "fp32_batched": {"value": r32, "unit": UNIT, **accuracy("fp32"), "tuning": out["fp32"]["tune"]},
        "mixed_batched": {"value": out["mixed"]["rate"], "unit": UNIT, **accuracy("mixed")},
        "fp64_batched": {"value": r64, "unit": UNIT},
        "fp64_strict_batched": {"value": r64s, "unit": UNIT},
        "fp64_one_at_a_time": {"value": one_rate, "unit": UNIT, "sample_instances": int(len(sample))},
        "fp32_batched_over_fp64_one_at_a_time": r32 / one_rate,
        "fp32_batched_over_fp64_batched": r32 / r64,
        "fp32_batched_over_fp64_strict_batched": r32 / r64s,
        "mixed_batched_over_fp64_one_at_a_time": out["mixed"]["rate"] / one_rate,
    }
    if e2e_rate is not None:
        summary["fp32_batched_e2e"] = {"value": e2e_rate, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                                       "d2h_bytes_per_step": nbytes, "ms_per_step": 1000.0 * e2e_s / steps}
    return summary, out


def run_gpu_batch(args, rank, world, local_rank):
    """The batched workload as the bench line: the FP32 batch over the window
    t in [0, C4_TEND] per step, against plain FP64 grids run one at a time."""
    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clocks = Clocks(local_rank)
    summary, out = batch_measure(args, world, dev, C4_TEND, args.steps, args.warmup, clocks, flush)
    head = out["fp32"]
    peak, peak_kind = measured_peaks()
    byts = 8.0 / 3.0 * 3 * 4
    gbs = byts * head["cells"] / (head["ms"] / 1000.0) / 1e9
    ck = clocks.summary()
    if rank == 0:
        e2e = summary.pop("fp32_batched_e2e")
        line = {"metric": METRIC, "value": summary["fp32_batched"]["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": summary["workload"], "cells_total": summary["cells_total"],
                           "instances": summary["instances"], "precision": "fp32", "tuning": head["tune"],
                           "l2": "flushed (256 MiB write) between timed steps",
                           "parallelism": "replicas (one independent batch per GPU)"},
                "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                             "traffic": None, "note": "whole batch step time (stage + controller kernels)",
                             "algorithmic_bytes_per_cell_stage": byts, "peak_source": peak_kind},
                "batched": summary, "cpu_baseline": None, "e2e": e2e,
                "gpu_launches": head["launches"], "clocks": ck}
        print(json.dumps(line), flush=True)
    for v in out.values():
        v["batch"].close()
    return 0


def _get_q_into(s, out):
    import ctypes
    from sharpclaw_b200 import _capi as C
    C.check(C.lib().scl_get_q(s._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "scl_get_q")
    return out


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp64", "fp64_strict"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-workload block of the default (c2) run")
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c3", "c4", "c5"],
                    help="c2 (default, the headline): 1-D Euler mx=2^20; c1 advection; c3 2-D shallow "
                         "water 4096^2; c4 2048 batched Euler Riemann problems; c5 2-D acoustics 1024^2")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "c4":
            return run_gpu_batch(args, rank, world, local_rank)
        return run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
