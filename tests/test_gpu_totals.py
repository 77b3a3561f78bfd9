"""Conserved totals kept on the device (scl_set_totals / scl_conserved_totals).

The totals kernel sums sum(q [* kappa]) * dx [* dy] of every component in
FP64 with compensated (error-free two-sum) accumulation, whatever the
arithmetic form of the stages.  Checked here:

* its values against the exactly rounded host sum (math.fsum) of the same
  state -- the initial one and the one the run ends with -- to a few ulps;
* on periodic grids with a conservative scheme (WENO5 + Godunov or Roe
  fluctuations with tfluct: the fluctuations telescope) the drift over a run
  is FP64 round-off in the FP64 forms, and the round-off of FP32 fluxes or
  FP32 state in the reduced-precision forms;
* a rejected step leaves the totals of the accepted state;
* the cluster-resident run keeps them too (summed by its tile code), equal
  to the graph run's to a few ulps.
"""
import math

import numpy as np
import pytest

import cases
import sharpclaw_b200 as S

pytestmark = pytest.mark.gpu

FORMS = ["fp64_strict", "fp64", "mixed", "fp32"]
# drift bound relative to sum |q| dx over the run, per form
DRIFT = {"fp64_strict": 1e-13, "fp64": 1e-13, "mixed": 2e-6, "fp32": 2e-5}


def _host_totals(q, ndim, area, kappa=None, fp32=False):
    if fp32:
        q = q.astype(np.float32).astype(np.float64)
        if kappa is not None:
            kappa = kappa.astype(np.float32).astype(np.float64)
    inner = q[:, 3:-3] if ndim == 1 else q[:, 3:-3, 3:-3]
    w = None if kappa is None else (kappa[3:-3] if ndim == 1 else kappa[3:-3, 3:-3])
    out = []
    for m in range(q.shape[0]):
        v = inner[m] if w is None else inner[m] * w
        out.append(math.fsum(v.ravel().tolist()) * area)
    scale = [math.fsum(np.abs(inner[m] if w is None else inner[m] * w).ravel().tolist()) * area
             for m in range(q.shape[0])]
    return np.array(out), np.array(scale)


@pytest.mark.parametrize("mode", [S.RUN_GRAPH, S.RUN_RESIDENT])
@pytest.mark.parametrize("precision", FORMS)
def test_periodic_advection_totals(precision, mode):
    po, ps, q, _ = cases.advection(mx=1000)
    ps.time_integrator = 3
    fp32 = precision == "fp32"
    with S.Solver(ps, precision) as s:
        s.set_run_mode(mode)
        s.set_totals(True)
        s.set_q(q)
        res = s.sharpclaw(0.0, 0.5, 0.0008, 0.85, 0.8)
        assert s.last_run()[0] == mode
        qf = s.get_q()
        T = s.conserved_totals()
    assert res["info"] == 0 and res["steps_taken"] > 500
    t0, scale = _host_totals(q, 1, ps.dx, fp32=fp32)
    t1, _ = _host_totals(qf, 1, ps.dx)
    assert np.all(np.abs(T["tot0"] - t0) <= 4e-16 * scale)
    assert np.all(np.abs(T["tot"] - t1) <= 4e-16 * scale)
    assert np.all(T["drift"] <= DRIFT[precision] * scale), (T["drift"] / scale)
    assert np.all(T["drift"] >= np.abs(T["tot"] - T["tot0"]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_periodic_shallow_water_2d_totals(precision):
    po, ps, q, _ = cases.radial_dam(n=64)
    ps.time_integrator = 3
    with S.Solver(ps, precision) as s:
        s.set_totals(True)
        s.set_q(q)
        res = s.time_steps(25, 0.004, 0.9, 0.8)[1]
        qf = s.get_q()
        T = s.conserved_totals()
    assert res["steps_taken"] == 25
    area = ps.dx * ps.dy
    t0, scale = _host_totals(q, 2, area)
    t1, _ = _host_totals(qf, 2, area)
    ref = scale[0]   # momenta sum to ~0: compare against the depth's magnitude
    assert np.all(np.abs(T["tot0"] - t0) <= 4e-16 * ref)
    assert np.all(np.abs(T["tot"] - t1) <= 4e-16 * ref)
    assert np.all(T["drift"] <= DRIFT[precision] * ref), T["drift"] / ref


def test_capacity_totals_weight_kappa():
    po, ps, q, aux = cases.with_capacity(cases.advection(mx=300))
    ps.time_integrator = 3
    kappa = aux[ps.mcapa - 1]
    with S.Solver(ps, "fp64") as s:
        s.set_aux(aux)
        s.set_totals(True)
        s.set_q(q)
        s.sharpclaw(0.0, 0.2, 0.001, 0.85, 0.8)
        qf = s.get_q()
        T = s.conserved_totals()
    t0, scale = _host_totals(q, 1, ps.dx, kappa)
    t1, _ = _host_totals(qf, 1, ps.dx, kappa)
    assert np.all(np.abs(T["tot0"] - t0) <= 4e-16 * scale)
    assert np.all(np.abs(T["tot"] - t1) <= 4e-16 * scale)
    assert np.all(T["drift"] <= 1e-13 * scale)


def test_rejected_step_keeps_the_accepted_totals():
    po, ps, q, _ = cases.shu_osher(mx=256, mthbc=(2, 2))
    ps.time_integrator = 3
    with S.Solver(ps, "fp64") as s:
        s.set_totals(True)
        s.set_q(q)
        res = s.sharpclaw(0.0, 0.01, 0.05, 0.9, 0.8)      # the first step is far too large
        qf = s.get_q()
        T = s.conserved_totals()
    assert res["rejected"] >= 1 and res["info"] == 0
    t1, scale = _host_totals(qf, 1, ps.dx)
    assert np.all(np.abs(T["tot"] - t1) <= 4e-16 * scale)


def test_resident_and_graph_totals_agree_with_capacity():
    po, ps, q, aux = cases.with_capacity(cases.advection(mx=500))
    ps.time_integrator = 4
    out = {}
    for mode in (S.RUN_GRAPH, S.RUN_RESIDENT):
        with S.Solver(ps, "fp64_strict") as s:
            s.set_run_mode(mode)
            s.set_aux(aux)
            s.set_totals(True)
            s.set_q(q)
            s.sharpclaw(0.0, 0.1, 0.001, 2.5, 2.4)
            assert s.last_run()[0] == mode
            out[mode] = (s.get_q(), s.conserved_totals())
    qg, Tg = out[S.RUN_GRAPH]
    qr, Tr = out[S.RUN_RESIDENT]
    assert np.array_equal(qg, qr)                      # the same arithmetic in both modes
    kappa = aux[ps.mcapa - 1]
    t1, scale = _host_totals(qr, 1, ps.dx, kappa)
    for T in (Tg, Tr):
        assert np.all(np.abs(T["tot"] - t1) <= 4e-16 * scale)
        assert np.all(T["drift"] <= 1e-13 * scale)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resident_totals_several_tiles_per_cta(precision):
    """5000 cells: 40 tiles on a cluster of 8, five per CTA; the CTA sums its
    tiles' warps in order, the controller warp the CTAs in rank order."""
    po, ps, q, _ = cases.advection(mx=5000)
    ps.time_integrator = 3
    with S.Solver(ps, precision) as s:
        s.set_run_mode(S.RUN_RESIDENT)
        s.set_totals(True)
        s.set_q(q)
        res = s.sharpclaw(0.0, 0.01, 0.0001, 0.85, 0.8)
        assert s.last_run()[0] == S.RUN_RESIDENT
        qf = s.get_q()
        T = s.conserved_totals()
    assert res["info"] == 0 and res["steps_taken"] > 10
    t0, scale = _host_totals(q, 1, ps.dx)
    t1, _ = _host_totals(qf, 1, ps.dx)
    assert np.all(np.abs(T["tot0"] - t0) <= 4e-16 * scale)
    assert np.all(np.abs(T["tot"] - t1) <= 4e-16 * scale)
    assert np.all(T["drift"] <= DRIFT[precision] * scale)


def test_totals_off_is_an_error():
    po, ps, q, _ = cases.advection(mx=200)
    with S.Solver(ps, "fp64") as s:
        with pytest.raises(S.SharpClawError):
            s.conserved_totals()
