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
