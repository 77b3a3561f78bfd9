"""Frame files in the reference's format (src/1d/out1.f90, src/2d/out2.f90),
written from host arrays through the C ABI (no GPU needed).

Pinned two ways: byte equality with the oracle's restatement of out1/out2,
and known answers of the Fortran E edit descriptor (Ew.d writes
[-]0.<d digits>E+xx, and +xxx without the E for three-digit exponents).
"""
import numpy as np
import pytest

import cases
from oracle import oracle as O
import sharpclaw_b200 as S


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def test_e_format_known_answers(tmp_path):
    vals = [1.0, -2.5, 0.0, 1.0e-5, 123456789.0, 1.0e100, 1.0e-120, -7.25e-99]
    mx = len(vals)
    q = np.zeros((1, mx + 6))
    q[0, 3:-3] = vals
    p = S.ClawParams(rp=S.RP_ADVECTION, mx=mx, dx=0.125, xlower=-5.0)
    S.write_frame(p, q, t=0.5, iframe=3, dir=str(tmp_path))
    lines = _read(tmp_path / "fort.q0003").decode().split("\n")
    assert lines[0] == "    1                 grid_number"
    assert lines[1] == "    1                 AMR_level"
    assert lines[2] == "    8                 mx"
    assert lines[3] == "   -0.50000000E+01    xlow"
    assert lines[4] == "    0.12500000E+00    dx"
    assert lines[5] == ""
    assert lines[6:14] == ["  0.10000000E+01", " -0.25000000E+01", "  0.00000000E+00", "  0.10000000E-04",
                           "  0.12345679E+09", "  0.10000000+101", "  0.00000000E+00", " -0.72500000E-98"]
    assert lines[14:] == ["  ", "  ", ""]
    t = _read(tmp_path / "fort.t0003").decode().split("\n")
    assert t == ["    0.5000000000000000E+00    time", "    1                 meqn",
                 "    1                 ngrids", "    0                 maux", "    1                 ndim",
                 "", "", ""]


def test_four_values_per_record(tmp_path):
    # meqn = 5 wraps after four values (format reversion of (4e16.8))
    mx = 3
    q = np.arange(5 * (mx + 6), dtype=np.float64).reshape(5, mx + 6) + 0.5
    p = S.ClawParams(rp=S.RP_ADVECTION, mx=mx, dx=0.1, meqn=5, mwaves=1)
    S.write_frame(p, q, t=1.0, iframe=7, dir=str(tmp_path))
    po = O.make_params(mx=mx, meqn=5, mwaves=1, dx=0.1, rp=O.RP_ADVECTION)
    ref = tmp_path / "ref"
    ref.mkdir()
    O.output(po, q, None, 1.0, 7, str(ref), False)
    got = _read(tmp_path / "fort.q0007")
    assert got == _read(ref / "fort.q0007")
    body = got.decode().split("\n")[6:]
    assert len(body[0]) == 64 and len(body[1]) == 16


@pytest.mark.parametrize("make,aux_out", [
    (lambda: cases.shu_osher(mx=50), False),
    (lambda: cases.radial_dam(n=9), True),
    (lambda: cases.acoustics2d(n=7), True),
])
def test_matches_oracle_restatement(tmp_path, make, aux_out):
    po, ps, q, aux = make()
    q = q.copy()
    q[(0,) + (3,) * (q.ndim - 2) + (slice(3, 5),)] = 1e-100   # written as 0
    S.write_frame(ps, q, aux, t=0.125, iframe=12345, dir=str(tmp_path), write_aux=aux_out)
    ref = tmp_path / "ref"
    ref.mkdir()
    O.output(po, q, aux, 0.125, 12345, str(ref), aux_out)
    names = ["fort.q2345", "fort.t2345"] + (["fort.a2345"] if aux_out and aux is not None else [])
    for n in names:
        assert _read(tmp_path / n) == _read(ref / n), n
    if not (aux_out and aux is not None):
        assert not (tmp_path / "fort.a2345").exists()


def test_bad_directory_is_an_error(tmp_path):
    p = S.ClawParams(rp=S.RP_ADVECTION, mx=4, dx=0.1)
    with pytest.raises(Exception):
        S.write_frame(p, np.zeros((1, 10)), t=0.0, iframe=0, dir=str(tmp_path / "missing"))
