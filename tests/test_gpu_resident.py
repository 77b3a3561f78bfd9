"""Cluster-resident runs of 1-D grids (the whole controller loop in one
launch) against the step graphs.

Both modes evaluate every interface and cell with the same tile code and the
same controller, so their results are bit-identical in every arithmetic form,
except the FP32 forms of 1-D Euler with char_decomp 0/2 and tfluct_solver 0,
whose graph path runs the paired kernel (two interfaces per thread in packed
FP32, a different contraction order): there the two agree to 1e-5 relative
after these short runs.  Bit-exactness against the oracle is covered by
test_gpu_parity.test_sharpclaw_run_strict in both modes.
"""
import numpy as np
import pytest

import cases
import sharpclaw_b200 as S

pytestmark = pytest.mark.gpu

CASES = [
    ("advection_cd0_tf1", lambda: cases.advection(mx=1000), 3, dict(tend=0.2, dt_initial=0.0008, cfl_max=0.85, cfl_desired=0.8)),
    ("advection_tvd2", lambda: cases.with_tvd(cases.advection(mx=300), (3, 1, 1, 1), 0), 3, dict(tend=0.2, dt_initial=0.002, cfl_max=0.85, cfl_desired=0.8)),
    ("euler_char_ssp104", lambda: cases.shu_osher(mx=400), 4, dict(tend=0.05, dt_initial=0.001, cfl_max=2.5, cfl_desired=2.45)),
    ("euler_comp_ssp33", lambda: cases.riemann(mx=250, char_decomp=0), 3, dict(tend=0.05, dt_initial=0.001, cfl_max=0.9, cfl_desired=0.8)),
    ("euler_wave", lambda: cases.riemann(mx=200, char_decomp=1), 4, dict(tend=0.05, dt_initial=0.001, cfl_max=2.5, cfl_desired=2.45)),
    ("acoustics_capa", lambda: cases.with_capacity(cases.acoustics1d(mx=150)), 3, dict(tend=0.3, dt_initial=0.002, cfl_max=0.9, cfl_desired=0.8)),
    ("acoustics_trans_wall_ssp22", lambda: cases.acoustics1d(mx=127, char_decomp=3, mthbc=(1, 3)), 1, dict(tend=0.3, dt_initial=0.002, cfl_max=0.9, cfl_desired=0.8)),
    # several tiles per CTA (40 tiles on a cluster of 8)
    ("advection_5000_ssp42", lambda: cases.advection(mx=5000), 2, dict(tend=0.02, dt_initial=0.0001, cfl_max=1.9, cfl_desired=1.8)),
    ("euler_5000", lambda: cases.shu_osher(mx=5000), 3, dict(tend=0.01, dt_initial=0.0001, cfl_max=0.9, cfl_desired=0.8)),
    # 1-D shallow water with the radial source term (src1.f90 of 1dRadialSymm-qwave)
    ("sw1d_radial_src", lambda: cases.radial_sw(mx=300), 4, dict(tend=0.2, dt_initial=0.002, cfl_max=1.0, cfl_desired=0.9)),
    # f-wave shallow water with neighbour aux in tfluct (1dPerturbSteady) and capacity (-kappa)
    ("swf_bathy", lambda: cases.fwave_bathymetry(mx=400), 4, dict(tend=0.02, dt_initial=0.0005, cfl_max=0.5, cfl_desired=0.2)),
    ("swf_kappa", lambda: cases.fwave_radial(mx=200, kappa=True), 4, dict(tend=0.01, dt_initial=0.001, cfl_max=0.3, cfl_desired=0.2)),
    # first step rejected and retaken
    ("euler_reject", lambda: cases.shu_osher(mx=120), 3, dict(tend=0.05, dt_initial=0.05, cfl_max=0.9, cfl_desired=0.8)),
    # a last chunk narrower than the halo: its left neighbour's row holds
    # ghost images too (periodic: 127 + 1 cells; two tiles per CTA, 1017
    # cells = 8 tiles of 127 + 1 cell on 5 CTAs; walls: 127 + 2 cells)
    ("advection_128_periodic", lambda: cases.advection(mx=128), 3, dict(tend=0.1, dt_initial=0.005, cfl_max=0.85, cfl_desired=0.8)),
    ("advection_1017_periodic", lambda: cases.advection(mx=1017), 4, dict(tend=0.01, dt_initial=0.001, cfl_max=2.5, cfl_desired=2.4)),
    ("acoustics_129_walls", lambda: cases.acoustics1d(mx=129, mthbc=(3, 3)), 3, dict(tend=0.2, dt_initial=0.002, cfl_max=0.9, cfl_desired=0.8)),
]


def _paired(ps, precision):
    return (ps.rp == S.RP_EULER and precision in ("mixed", "fp32") and ps.char_decomp in (0, 2)
            and ps.tfluct_solver == 0 and ps.lim_type == 2 and ps.mcapa == 0)


def _run(ps, q, aux, precision, mode, run, **kw):
    with S.Solver(ps, precision) as s:
        s.set_run_mode(mode)
        s.set_aux(aux) if aux is not None else None
        s.set_q(q)
        res = s.sharpclaw(0.0, run["tend"], run["dt_initial"], run["cfl_max"], run["cfl_desired"], **kw)
        return s.get_q(), res, s.last_run()


@pytest.mark.parametrize("precision", ["fp64_strict", "fp64", "mixed", "fp32"])
@pytest.mark.parametrize("name,make,ti,run", CASES, ids=[c[0] for c in CASES])
def test_resident_matches_graph(name, make, ti, run, precision):
    po, ps, q, aux = make()
    ps.time_integrator = ti
    qg, rg, lg = _run(ps, q, aux, precision, S.RUN_GRAPH, run)
    qr, rr, lr = _run(ps, q, aux, precision, S.RUN_RESIDENT, run)
    assert lg[0] == S.RUN_GRAPH and lr[0] == S.RUN_RESIDENT
    assert lr[1] == 1          # fewer than 4096 controller iterations: one launch
    assert lg[1] > 10 * rg["steps_taken"] // 2
    assert rg["steps_taken"] > 0
    if name == "euler_reject":
        assert rg["rejected"] >= 1
    if _paired(ps, precision):
        assert rr["steps_taken"] == rg["steps_taken"] and rr["rejected"] == rg["rejected"]
        for m in range(qg.shape[0]):
            err = np.abs(qr[m, 3:-3] - qg[m, 3:-3]).max() / np.abs(qg[m, 3:-3]).max()
            assert err <= 1e-5, (m, err)
        return
    assert rr == rg
    assert np.array_equal(qr[:, 3:-3], qg[:, 3:-3])


def test_resident_relaunch():
    """More controller iterations than one resident launch runs (4096): the
    host relaunches until the controller is done; the result equals the
    graphs' bit for bit."""
    po, ps, q, aux = cases.advection(mx=40)
    ps.time_integrator = 3
    run = dict(tend=80.0, dt_initial=0.01, cfl_max=0.85, cfl_desired=0.3)   # dt = 0.0075: 10667 steps
    qg, rg, _ = _run(ps, q, aux, "fp64_strict", S.RUN_GRAPH, run)
    qr, rr, lr = _run(ps, q, aux, "fp64_strict", S.RUN_RESIDENT, run)
    assert rg["steps_taken"] > 2 * 4096
    # the step that reaches tend sets done in the launch that takes it
    assert lr == (S.RUN_RESIDENT, -(-rg["steps_taken"] // 4096))
    assert rr == rg
    assert np.array_equal(qr[:, 3:-3], qg[:, 3:-3])


def test_resident_max_steps():
    """max_steps stops a resident run exactly where it stops the graphs
    (info = too many steps)."""
    po, ps, q, aux = cases.advection(mx=500)
    ps.time_integrator = 3
    run = dict(tend=1.0, dt_initial=0.001, cfl_max=0.85, cfl_desired=0.8)
    qg, rg, _ = _run(ps, q, aux, "fp64", S.RUN_GRAPH, run, max_steps=37)
    qr, rr, _ = _run(ps, q, aux, "fp64", S.RUN_RESIDENT, run, max_steps=37)
    assert rg["steps_taken"] == 37 and rg["info"] == S.C.INFO_TOO_MANY_STEPS
    assert rr == rg
    assert np.array_equal(qr, qg)


def test_auto_mode():
    """RUN_AUTO: resident for 1-D grids of at most 8 tiles of 127 cells (one
    per CTA), graphs for larger grids and for 2-D grids."""
    run = dict(tend=0.001, dt_initial=0.0001, cfl_max=0.85, cfl_desired=0.8)
    for mx, want in ((1016, S.RUN_RESIDENT), (1017, S.RUN_GRAPH)):
        _, ps, q, aux = cases.advection(mx=mx)
        assert _run(ps, q, aux, "fp64", S.RUN_AUTO, run)[2][0] == want
    _, ps, q, aux = cases.radial_dam(n=24)
    assert _run(ps, q, aux, "fp64", S.RUN_AUTO, dict(tend=0.01, dt_initial=0.001, cfl_max=0.9,
                                                     cfl_desired=0.8))[2][0] == S.RUN_GRAPH


def test_run_mode_errors():
    _, ps, q, aux = cases.radial_dam(n=16)
    with S.Solver(ps, "fp64") as s:
        with pytest.raises(S.SharpClawError):
            s.set_run_mode(S.RUN_RESIDENT)          # 2-D
        with pytest.raises(S.SharpClawError):
            s.set_run_mode(7)
        s.set_run_mode(S.RUN_GRAPH)
    _, ps, q, aux = cases.advection(mx=64 * 127 + 1)
    with S.Solver(ps, "fp64") as s:
        with pytest.raises(S.SharpClawError):
            s.set_run_mode(S.RUN_RESIDENT)          # 65 tiles
    _, ps, q, aux = cases.advection(mx=64 * 127)
    with S.Solver(ps, "fp64") as s:
        s.set_run_mode(S.RUN_RESIDENT)
