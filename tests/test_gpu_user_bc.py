"""The stegoton's hooks on a GPU: its b4step1.f time reversal
(SCL_B4STEP_TIME_REVERSAL) and the user boundary condition of
apps/elasticity/stegoton/bc1.f
(SCL_BC_USER_OSCILLATING_WALL): an oscillating wall at xlower (mthbc 0)
driven at each stage's time, extrapolation at xupper, and the switch of both
sides to periodic once a stage time enters (5 tw1, 5 tw1 + 1).  Compared with
the oracle (oracle/sclaw_oracle.c bc1_user) one step at a time and over whole
runs across the switch; the stress law exp(K eps) - 1 and the wall's cos are
evaluated by the device's and the host's libm, so results agree to rounding
(1e-11 relative) rather than bit for bit."""
import numpy as np
import pytest

import cases
import sharpclaw_b200 as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {"fp64_strict": 1e-11, "fp64": 1e-10, "mixed": 2e-5, "fp32": 2e-4}


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64", "mixed", "fp32"])
@pytest.mark.parametrize("t", [0.4, 1.3, 5.5])   # wall moving, near its peak, inside the switch window
def test_step_parity(t, precision):
    po, ps, q, aux = cases.stegoton_wall(mx=96)
    rng = np.random.default_rng(11)
    q = 0.02 * rng.standard_normal(q.shape)
    dt = 0.5 * po.dx
    _, dqo, cflo = O.step(po, q, aux, dt, t)
    with S.Solver(ps, precision) as s:
        s.set_aux(aux)
        _, dq, cfl = s.step(q, dt, t)
    assert _rel(dq[:, 3:-3], dqo[:, 3:-3]) <= TOL[precision]
    assert abs(cfl - cflo) <= max(TOL[precision], 1e-6) * cflo


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64"])
@pytest.mark.parametrize("ti", [3, 4])
def test_run_across_the_switch(ti, precision):
    """From rest to t = 5.6 (the wall pulse, its travel, the switch), then on to
    t = 6.4 in a second call: the switch is remembered by the handle, as
    bc1.f's rewrite of mthbc is by ClawParams."""
    po, ps, q, aux = cases.stegoton_wall(mx=288)
    ps.time_integrator = ti
    cfl = (2.5, 2.45) if ti == 4 else (0.9, 0.8)
    run = dict(dt_initial=0.01, cfl_max=cfl[0], cfl_desired=cfl[1])
    qo, ro = O.sharpclaw(po, q, aux, tstart=0.0, tend=5.6, time_integrator=ti, **run)
    assert ro.bc_switched == 1 and ro.info == 0
    with S.Solver(ps, precision) as s:
        s.set_aux(aux)
        s.set_q(q)
        res = s.sharpclaw(0.0, 5.6, run["dt_initial"], run["cfl_max"], run["cfl_desired"])
        assert s.last_run()[0] == S.RUN_GRAPH     # the hook keeps runs off the resident path
        q1 = s.get_q()
        assert res["steps_taken"] == ro.steps_taken and res["rejected"] == ro.rejected
        assert res["info"] == 0
        assert _rel(q1[:, 3:-3], qo[:, 3:-3]) <= 10 * TOL[precision]
        # second call, continuing from the device state
        po2 = cases.stegoton_wall(mx=288)[0]
        po2.bc_switched = 1
        qo2, ro2 = O.sharpclaw(po2, qo, aux, tstart=5.6, tend=6.4, time_integrator=ti, **run)
        res2 = s.sharpclaw(5.6, 6.4, run["dt_initial"], run["cfl_max"], run["cfl_desired"])
        q2 = s.get_q()
    assert res2["steps_taken"] == ro2.steps_taken
    assert _rel(q2[:, 3:-3], qo2[:, 3:-3]) <= 10 * TOL[precision]
    # periodic from the switch on: the resting wall and extrapolation of a
    # run without the switch end elsewhere
    po3 = cases.stegoton_wall(mx=288, mthbc=(3, 1))[0]
    po3.bc_user = 0
    qo3, _ = O.sharpclaw(po3, qo, aux, tstart=5.6, tend=6.4, time_integrator=ti, **run)
    if _rel(qo3[:, 3:-3], qo2[:, 3:-3]) < 1e-9:
        pytest.fail("the switch made no difference: the case does not exercise it")


def test_user_bc_refused_where_not_built():
    po, ps, q, aux = cases.stegoton_wall(mx=96)
    with S.Solver(ps, "fp64") as s:
        with pytest.raises(S.SharpClawError):
            s.set_run_mode(S.RUN_RESIDENT)
            s.set_aux(aux)
            s.set_q(q)
            s.sharpclaw(0.0, 0.1, 0.01, 2.5, 2.45)


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64"])
def test_time_reversal_run_parity(precision):
    """Layered medium, strain 0.02 (nonlinear), periodic, variable dt: the flip
    at the first step from t = 2.5 on, then a second call that must not flip
    again (itrdone of /comtimereverse/ is kept by the handle)."""
    po, ps, q, aux = cases.stegoton(mx=400, amp=0.02, mthbc=(2, 2))
    ps.time_integrator = 4
    run = dict(dt_initial=0.01, cfl_max=2.5, cfl_desired=2.45)
    po.b4step, po.trtime = 2, 2.5
    qo, ro = O.sharpclaw(po, q, aux, tstart=0.0, tend=5.0, time_integrator=4, **run)
    po.b4_done = 1
    qo2, ro2 = O.sharpclaw(po, qo, aux, tstart=5.0, tend=6.0, time_integrator=4, **run)
    with S.Solver(ps, precision) as s:
        s.set_aux(aux)
        s.set_b4step(S.B4STEP_TIME_REVERSAL, 2.5)
        s.set_q(q)
        res = s.sharpclaw(0.0, 5.0, run["dt_initial"], run["cfl_max"], run["cfl_desired"])
        q1 = s.get_q()
        res2 = s.sharpclaw(5.0, 6.0, run["dt_initial"], run["cfl_max"], run["cfl_desired"])
        q2 = s.get_q()
    assert res["steps_taken"] == ro.steps_taken and res2["steps_taken"] == ro2.steps_taken
    assert _rel(q1[:, 3:-3], qo[:, 3:-3]) <= 10 * TOL[precision]
    assert _rel(q2[:, 3:-3], qo2[:, 3:-3]) <= 10 * TOL[precision]


def test_time_reversal_restores_the_pulse():
    """The known answer of the oracle test on the device, in the FMA form."""
    _, ps, q, _ = cases.stegoton(mx=600, amp=1e-4, mthbc=(2, 2))
    aux = np.ascontiguousarray(np.stack([np.ones(606), np.ones(606), np.zeros(606)]))
    ps.time_integrator = 4
    with S.Solver(ps, "fp64") as s:
        s.set_aux(aux)
        s.set_b4step(S.B4STEP_TIME_REVERSAL, 5.0)
        s.set_q(q)
        r = s.sharpclaw(0.0, 10.0, 1 / 32, 2.5, 2.45, dt_variable=0)
        qf = s.get_q()
    scale = np.abs(q[0, 3:-3]).max()
    assert r["info"] == 0
    assert np.abs(qf[0, 3:-3] - q[0, 3:-3]).max() <= 2e-6 * scale


def test_time_reversal_restores_the_pulse_mixed():
    """The same in the mixed form, whose FP32 stress is expm1f(K eps): no
    cancellation at strain 1e-4 (exp(K eps) - 1 in FP32 left a 1.1e-2 error;
    expm1f gives 5.0e-7, as FP64)."""
    _, ps, q, _ = cases.stegoton(mx=600, amp=1e-4, mthbc=(2, 2))
    aux = np.ascontiguousarray(np.stack([np.ones(606), np.ones(606), np.zeros(606)]))
    ps.time_integrator = 4
    with S.Solver(ps, "mixed") as s:
        s.set_aux(aux)
        s.set_b4step(S.B4STEP_TIME_REVERSAL, 5.0)
        s.set_q(q)
        r = s.sharpclaw(0.0, 10.0, 1 / 32, 2.5, 2.45, dt_variable=0)
        qf = s.get_q()
    scale = np.abs(q[0, 3:-3]).max()
    assert r["info"] == 0
    assert np.abs(qf[0, 3:-3] - q[0, 3:-3]).max() <= 2e-6 * scale
