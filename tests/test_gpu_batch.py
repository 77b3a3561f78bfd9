"""GPU tests of the batched solver (scl_batch_*): every instance of a batch of
uneven problems must evolve exactly as the oracle's sharpclaw() on that
problem alone -- bit for bit in FP64_STRICT, including rejected and retaken
steps and per-instance final times -- and the FP32 batch must stay close to
the FP64 oracle."""
import numpy as np
import pytest

import cases
from oracle import oracle as O
import sharpclaw_b200 as S

pytestmark = pytest.mark.gpu


def _euler_batch(seed, mxs):
    rng = np.random.default_rng(seed)
    probs = []
    for mx in mxs:
        rho = rng.uniform(0.1, 1.0, 2)
        u = rng.uniform(-1.0, 1.0, 2)
        p = rng.uniform(0.1, 1.0, 2)
        po, ps, q, _ = cases.riemann(mx=int(mx), rho=tuple(rho), u=tuple(u), p=tuple(p))
        c = np.sqrt(1.4 * p / rho)
        smax = float(np.max(np.abs(u) + c))
        probs.append((po, q, 1.0 / mx, smax))
    return probs


def test_batch_euler_strict_matches_oracle_per_instance():
    mxs = [40, 129, 300, 777, 64, 1000, 33, 256]
    probs = _euler_batch(4, mxs)
    ps = S.ClawParams(rp=S.RP_EULER, mx=10, dx=0.1, mthbc=(1, 1), char_decomp=0, tfluct_solver=0,
                      time_integrator=3)
    tend, cfl_max, cfl_des = 0.05, 0.9, 0.8
    # instance 2 starts with a step far too large: rejected, then retaken
    dt0 = np.array([cfl_des * dx / sm for (_, _, dx, sm) in probs])
    dt0[2] *= 4.0
    with S.Batch(ps, mxs, [p[2] for p in probs], precision="fp64_strict") as b:
        b.set_q([p[1] for p in probs])
        res, ms = b.sharpclaw(0.0, tend, dt0, cfl_max, cfl_des)
        got = b.get_q()
    assert ms > 0
    for k, (po, q, dx, sm) in enumerate(probs):
        qo, ro = O.sharpclaw(po, q, None, tstart=0.0, tend=tend, dt_initial=float(dt0[k]), cfl_max=cfl_max,
                             cfl_desired=cfl_des, time_integrator=3)
        r = res[k]
        assert (r["steps_taken"], r["rejected"], r["info"]) == (ro.steps_taken, ro.rejected, ro.info), k
        assert r["tend"] == ro.tend and r["dt_last"] == ro.dt_last and r["cfl_maxused"] == ro.cfl_maxused
        assert np.array_equal(got[k][:, 3:-3], qo[:, 3:-3]), k
    assert res[2]["rejected"] >= 1


def test_batch_advection_tfluct_strict_and_rerun():
    mxs = [50, 200, 333]
    qs, pos = [], []
    for mx in mxs:
        po, ps, q, _ = cases.advection(mx=mx)
        qs.append(q)
        pos.append(po)
    ps = S.ClawParams(rp=S.RP_ADVECTION, mx=10, dx=0.1, mthbc=(2, 2), char_decomp=0, tfluct_solver=1,
                      time_integrator=4)
    dxs = [1.0 / m for m in mxs]
    with S.Batch(ps, mxs, dxs, precision="fp64_strict") as b:
        b.set_q(qs)
        res1, _ = b.sharpclaw(0.0, 0.1, [0.5 * d for d in dxs], 2.5, 2.4)
        res2, _ = b.sharpclaw(0.1, 0.2, [0.5 * d for d in dxs], 2.5, 2.4)   # continue from the state
        got = b.get_q()
    for k, po in enumerate(pos):
        q1, r1 = O.sharpclaw(po, qs[k], None, tstart=0.0, tend=0.1, dt_initial=0.5 * dxs[k], cfl_max=2.5,
                             cfl_desired=2.4, time_integrator=4)
        q2, r2 = O.sharpclaw(po, q1, None, tstart=0.1, tend=0.2, dt_initial=0.5 * dxs[k], cfl_max=2.5,
                             cfl_desired=2.4, time_integrator=4)
        assert res1[k]["steps_taken"] == r1.steps_taken and res2[k]["steps_taken"] == r2.steps_taken
        assert np.array_equal(got[k][:, 3:-3], q2[:, 3:-3])


@pytest.mark.parametrize("variant", [-1, 0, 1, 2])
@pytest.mark.parametrize("precision,tol", [("fp32", 2e-5), ("mixed", 2e-5)])
def test_batch_euler_reduced_precision(precision, tol, variant):
    mxs = [100, 400, 250]
    probs = _euler_batch(9, mxs)
    ps = S.ClawParams(rp=S.RP_EULER, mx=10, dx=0.1, mthbc=(1, 1), char_decomp=0, tfluct_solver=0,
                      time_integrator=3)
    dt0 = [0.5 * dx / sm for (_, _, dx, sm) in probs]
    with S.Batch(ps, mxs, [p[2] for p in probs], precision=precision) as b:
        b.select(variant)      # 0, 1: one interface per thread; 2: two (Euler FP32 forms)
        b.set_q([p[1] for p in probs])
        res, _ = b.sharpclaw(0.0, 0.05, dt0, 0.9, 0.8)
        got = b.get_q()
        tune = b.tuning()
    assert tune["threads"] in (128, 256) and tune["grid"] > 0
    assert variant < 0 or tune["variant"] == variant
    for k, (po, q, dx, sm) in enumerate(probs):
        qo, ro = O.sharpclaw(po, q, None, tstart=0.0, tend=0.05, dt_initial=dt0[k], cfl_max=0.9, cfl_desired=0.8,
                             time_integrator=3)
        assert res[k]["tend"] == pytest.approx(0.05)
        for m in range(3):
            rel = np.abs(got[k][m, 3:-3] - qo[m, 3:-3]).sum() / np.abs(qo[m, 3:-3]).sum()
            assert rel <= tol, (k, m, rel)
