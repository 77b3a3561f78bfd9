"""Frame files written from the device state (scl_write_frame): the copy is
enqueued on the handle's stream and a host thread writes the files, so the
files must equal those written from a host copy of the same state, even when
the device has advanced since."""
import numpy as np
import pytest

import cases
import sharpclaw_b200 as S

pytestmark = pytest.mark.gpu


def _read(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("make,precision", [
    (lambda: cases.shu_osher(mx=120), "fp32"),      # FP32 storage: converted on the device
    (lambda: cases.acoustics2d(n=20), "mixed"),     # 2-D, aux written (the 2-D default)
])
def test_device_frame_equals_host_frame(tmp_path, make, precision):
    po, ps, q, aux = make()
    with S.Solver(ps, precision) as s:
        s.set_aux(aux) if aux is not None else None
        s.set_q(q)
        dt = 0.2 * (ps.dx if ps.rp != S.RP_EULER else ps.dx / 5.0)
        s.rk_step(dt)
        q1 = s.get_q()
        s.write_frame(0.25, 4, dir=str(tmp_path))
        for _ in range(3):           # the device moves on while the frame is written
            s.rk_step(dt)
        s.wait_frames()
        q4 = s.get_q()
    assert not np.array_equal(q1, q4)
    ref = tmp_path / "ref"
    ref.mkdir()
    S.write_frame(ps, q1, aux, t=0.25, iframe=4, dir=str(ref))
    names = ["fort.q0004", "fort.t0004"] + (["fort.a0004"] if ps.ndim == 2 else [])
    for n in names:
        assert _read(tmp_path / n) == _read(ref / n), n


def test_write_error_is_reported_on_wait(tmp_path):
    po, ps, q, aux = cases.advection(mx=64)
    with S.Solver(ps, "fp64") as s:
        s.set_q(q)
        s.write_frame(0.0, 0, dir=str(tmp_path / "missing"))
        with pytest.raises(Exception):
            s.wait_frames()
        s.write_frame(0.0, 1, dir=str(tmp_path))     # the handle stays usable
        s.wait_frames()
    assert (tmp_path / "fort.q0001").exists()


@pytest.mark.parametrize("make,ti,run", [
    (lambda: cases.acoustics1d(mx=100), 4, dict(dt_initial=0.025, cfl_max=2.9, cfl_desired=2.85, tfinal=2.0, nout=4)),
    (lambda: cases.radial_dam(n=24), 3, dict(dt_initial=0.01, cfl_max=0.9, cfl_desired=0.8, tfinal=0.3, nout=3)),
])
def test_run_frames_matches_the_reference_driver(tmp_path, make, ti, run):
    """Solver.run_frames follows main.f90's output loop: the frames it writes
    from the device (FP64_STRICT) are byte-identical to the oracle run through
    the same loop (sharpclaw per interval, dt_initial = dt_last, out1/out2)."""
    from oracle import oracle as O
    po, ps, q, aux = make()
    ps.time_integrator = ti
    gdir, odir = tmp_path / "gpu", tmp_path / "oracle"
    gdir.mkdir()
    odir.mkdir()
    with S.Solver(ps, "fp64_strict") as s:
        s.set_aux(aux) if aux is not None else None
        s.set_q(q)
        res = s.run_frames(0.0, run["dt_initial"], run["cfl_max"], run["cfl_desired"], nout=run["nout"],
                           tfinal=run["tfinal"], outdir=str(gdir))
    outaux = ps.ndim == 2
    qo = O.bc(po, q)
    O.output(po, qo, aux, 0.0, 0, str(odir), outaux)
    dt, tend = run["dt_initial"], 0.0
    dtout = run["tfinal"] / run["nout"]
    for n in range(1, run["nout"] + 1):
        tstart, tend = tend, tend + dtout
        qo, ro = O.sharpclaw(po, qo, aux, tstart=tstart, tend=tend, dt_initial=dt, cfl_max=run["cfl_max"],
                             cfl_desired=run["cfl_desired"], time_integrator=ti)
        assert res[n - 1]["steps_taken"] == ro.steps_taken and res[n - 1]["info"] == ro.info
        dt = ro.dt_last
        O.output(po, qo, aux, tend, n, str(odir), outaux)
    names = sorted(p.name for p in odir.iterdir())
    assert names == sorted(p.name for p in gdir.iterdir())
    assert len(names) == (run["nout"] + 1) * (3 if outaux and ps.maux > 0 else 2)
    for name in names:
        assert _read(gdir / name) == _read(odir / name), name
