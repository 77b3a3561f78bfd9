"""GPU parity at the benchmark configurations' full sizes, against the oracle.

The other parity tests use grids the oracle steps in milliseconds; these run
the oracle (C, one core, or a spawned pool) at the sizes the benchmarks use,
so that the size-dependent parts of the device path are compared too: the
64-bit plane and pitch offsets of 4096^2 grids, tens of thousands of CTAs
per stage and their CFL atomics, the batched solver's tile -> instance
search over 2048 instances of up to 65,536 cells, and a whole run's
controller loop.  Workloads (synthetic, seeded, the benchmark's recipes):

  1-D Euler Shu-Osher, mx = 2^20, Roe + entropy fix, char-wise WENO5,
      tfluct_solver 0: one SSPRK(10,4) step and one dq evaluation;
  2-D shallow water, 4096^2 radial dam + N(0, 1e-3) noise, periodic,
      char-wise WENO5, tfluct: one stage (dq = dt L(q), flux2);
  1-D advection, mx = 1000, the whole run to t = 1 (SSPRK(3,3), cfl 0.8/0.85),
      in step graphs and in one cluster-resident launch;
  2048 batched 1-D Euler Riemann problems (mx log-uniform in [256, 65536],
      seed 4): a window t in [0, 5e-4], 32 sampled instances (the largest
      included) against the oracle's sharpclaw() one by one;
  2-D variable-coefficient acoustics, 1024^2, smoothed log-normal rho, K:
      one SSPRK(3,3) step.

FP64_STRICT must equal the oracle bit for bit; FP64 within 1e-12 relative
L-infinity (dq normalised by max |dq|); the FP32 forms within the 1e-5
relative L1 bound the reduced-precision forms are specified with.
"""
import multiprocessing as mp

import numpy as np
import pytest

import bench
import cases
from oracle import oracle as O
import sharpclaw_b200 as S

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_L1_FP32 = 1e-5


def _rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _rel_l1(a, b):
    return max(float(np.abs(a[m] - b[m]).sum() / max(np.abs(b[m]).sum(), 1e-300)) for m in range(a.shape[0]))


# ---- 1-D Euler, mx = 2^20 ----------------------------------------------------
@pytest.fixture(scope="module")
def c2_oracle():
    po, ps, q, _ = cases.shu_osher(mx=bench.MX)
    ps.time_integrator = 4
    qb = O.bc(po, q)
    ref, cfl = O.rk_step(po, 4, qb, None, bench.DT0)
    return po, ps, q, ref, cfl


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64", "mixed", "fp32"])
def test_euler_2p20_ssp104_step(c2_oracle, precision):
    po, ps, q, ref, cflr = c2_oracle
    with S.Solver(ps, precision) as s:
        s.set_q(q)
        cfl = s.rk_step(bench.DT0)
        got = s.get_q()
    a, b = got[:, 3:-3], ref[:, 3:-3]
    if precision == "fp64_strict":
        assert np.array_equal(a, b), f"max |diff| {np.abs(a - b).max()}"
        assert cfl == cflr
    elif precision == "fp64":
        assert _rel_inf(a, b) <= TOL_FP64
        assert abs(cfl - cflr) <= TOL_FP64 * cflr
    else:
        assert _rel_l1(a, b) <= TOL_L1_FP32
        assert abs(cfl - cflr) <= 1e-5 * cflr


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64"])
def test_euler_2p20_dq(precision):
    po, ps, q, _ = cases.shu_osher(mx=bench.MX)
    qo, dqo, cflo = O.step(po, q, None, bench.DT0)
    with S.Solver(ps, precision) as s:
        qg, dqg, cflg = s.step(q, bench.DT0)
    assert np.array_equal(qg, qo)
    a, b = dqg[:, 3:-3], dqo[:, 3:-3]
    if precision == "fp64_strict":
        assert np.array_equal(a, b) and cflg == cflo
    else:
        assert np.abs(a - b).max() <= TOL_FP64 * np.abs(b).max()
        assert abs(cflg - cflo) <= TOL_FP64 * cflo


# ---- 2-D shallow water, 4096^2 -----------------------------------------------
@pytest.fixture(scope="module")
def c3_oracle():
    po, ps, q, _ = cases.radial_dam(n=4096)
    dt = 0.3 * ps.dx / 1.5
    qo, dqo, cflo = O.step(po, q, None, dt)
    return ps, q, dt, qo, dqo, cflo


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64", "mixed"])
def test_shallow_water_4096_stage(c3_oracle, precision):
    ps, q, dt, qo, dqo, cflo = c3_oracle
    with S.Solver(ps, precision) as s:
        qg, dqg, cflg = s.step(q, dt)
    assert np.array_equal(qg, qo), "ghost-cell fill differs from bc2"
    a, b = dqg[:, 3:-3, 3:-3], dqo[:, 3:-3, 3:-3]
    if precision == "fp64_strict":
        assert np.array_equal(a, b), f"max |diff| {np.abs(a - b).max()}"
        assert cflg == cflo
    elif precision == "fp64":
        assert np.abs(a - b).max() <= TOL_FP64 * np.abs(b).max()
        assert abs(cflg - cflo) <= TOL_FP64 * cflo
    else:
        # one stage's dq from FP32 reconstructions and Riemann solves
        assert _rel_l1(a, b) <= 1e-4
        assert abs(cflg - cflo) <= 1e-5 * cflo


# ---- 1-D advection, mx = 1000, the whole run ----------------------------------
@pytest.mark.parametrize("mode", ["graph", "resident"])
def test_advection_1000_full_run(mode):
    po, ps, q, _ = cases.advection(mx=1000)
    ps.time_integrator = 3
    run = dict(tend=1.0, dt_initial=0.8 / 1000, cfl_max=0.85, cfl_desired=0.8)
    qo, ro = O.sharpclaw(po, q, None, tstart=0.0, time_integrator=3, **run)
    with S.Solver(ps, "fp64_strict") as s:
        s.set_run_mode(S.RUN_GRAPH if mode == "graph" else S.RUN_RESIDENT)
        s.set_q(q)
        res = s.sharpclaw(0.0, run["tend"], run["dt_initial"], run["cfl_max"], run["cfl_desired"])
        qg = s.get_q()
        assert s.last_run()[0] == (S.RUN_GRAPH if mode == "graph" else S.RUN_RESIDENT)
    assert ro.steps_taken > 1000 and ro.info == 0
    assert (res["steps_taken"], res["rejected"], res["info"]) == (ro.steps_taken, ro.rejected, ro.info)
    assert res["tend"] == ro.tend and res["dt_last"] == ro.dt_last and res["cfl_maxused"] == ro.cfl_maxused
    assert np.array_equal(qg[:, 3:-3], qo[:, 3:-3])


# ---- 2048 batched Riemann problems ---------------------------------------------
C4_WINDOW = 5e-4
C4_CFL = (0.9, 0.8)


@pytest.fixture(scope="module")
def c4_sample():
    mx, dx, qs, dt0 = bench.c4_instances()
    rng = np.random.default_rng(444)
    sample = sorted(set(rng.choice(len(mx), 31, replace=False).tolist()) | {int(np.argmax(mx))})
    jobs = [(int(mx[k]), float(dx[k]), qs[k], float(dt0[k]), C4_WINDOW, C4_CFL) for k in sample]
    with mp.get_context("spawn").Pool(min(16, len(jobs))) as pool:
        ref = pool.map(cases.oracle_riemann_window, jobs)
    return mx, dx, qs, dt0, sample, ref


def _c4_params():
    return S.ClawParams(rp=S.RP_EULER, mx=10, dx=0.1, mthbc=(1, 1), char_decomp=0, tfluct_solver=0,
                        time_integrator=3, gamma=bench.GAMMA)


def test_batch_2048_strict_sampled_instances(c4_sample):
    mx, dx, qs, dt0, sample, ref = c4_sample
    assert int(np.argmax(mx)) in sample and int(mx.max()) > 60000
    with S.Batch(_c4_params(), mx, dx, precision="fp64_strict") as b:
        b.set_q(qs)
        res, _ = b.sharpclaw(0.0, C4_WINDOW, dt0, *C4_CFL)
        got = b.get_q()
    for k, (qo, ro) in zip(sample, ref):
        r = res[k]
        assert (r["steps_taken"], r["rejected"], r["info"]) == (ro["steps_taken"], ro["rejected"], ro["info"]), k
        assert r["tend"] == ro["tend"] and r["dt_last"] == ro["dt_last"] and r["cfl_maxused"] == ro["cfl_maxused"]
        assert np.array_equal(got[k][:, 3:-3], qo[:, 3:-3]), k


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_batch_2048_reduced_precision_sampled_instances(c4_sample, precision):
    mx, dx, qs, dt0, sample, ref = c4_sample
    with S.Batch(_c4_params(), mx, dx, precision=precision) as b:
        b.set_q(qs)
        res, _ = b.sharpclaw(0.0, C4_WINDOW, dt0, *C4_CFL)
        got = b.get_q()
    for k, (qo, ro) in zip(sample, ref):
        if ro["info"] != 0:
            continue
        assert res[k]["info"] == 0 and res[k]["tend"] == pytest.approx(C4_WINDOW)
        assert _rel_l1(got[k][:, 3:-3], qo[:, 3:-3]) <= TOL_L1_FP32, k


# ---- 2-D acoustics, 1024^2 ----------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64_strict", "fp64"])
def test_acoustics_1024_ssp33_step(precision):
    W = bench.workloads()["c5"]()
    ps, q, aux, dt = W["params"], W["q"], W["aux"], W["dt0"]
    po = O.make_params(ndim=2, meqn=3, mwaves=2, maux=2, rp=O.RP_ACOUSTICS2D, mx=ps.mx, my=ps.my, dx=ps.dx,
                       dy=ps.dy, mthbc=(2, 2, 2, 2), char_decomp=0, tfluct_solver=1)
    ref, cflr = O.rk_step(po, 3, O.bc(po, q), aux, dt)
    with S.Solver(ps, precision) as s:
        s.set_aux(aux)
        s.set_q(q)
        cfl = s.rk_step(dt)
        got = s.get_q()
    a, b = got[:, 3:-3, 3:-3], ref[:, 3:-3, 3:-3]
    if precision == "fp64_strict":
        assert np.array_equal(a, b) and cfl == cflr
    else:
        assert _rel_inf(a, b) <= TOL_FP64
        assert abs(cfl - cflr) <= TOL_FP64 * cflr
