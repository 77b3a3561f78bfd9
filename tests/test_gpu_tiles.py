"""2-D tile shapes of the fused stage kernel.

Every shape evaluates each interface and each cell with the same source
arithmetic.  In FP64_STRICT (no FMA contraction) full runs with any fixed
shape, and with the shape the autotuner picks, agree bit for bit and equal the
oracle.  In the forms compiled with FMA contraction the compiler may fuse a
different product of a sum such as a*b + c*d in each kernel instantiation, so
shapes agree to the rounding of that form: 1e-13 relative (FP64), 1e-6
relative (FP32 reconstruction, after about 20 steps).
"""
import numpy as np
import pytest

import cases
from oracle import oracle as O
import sharpclaw_b200 as S

pytestmark = pytest.mark.gpu

RUN = dict(tend=0.3, dt_initial=0.004, cfl_max=0.5, cfl_desired=0.45)

TILE_CASES = [
    ("sw2d_char_tf1", lambda: cases.radial_dam(n=45)),
    ("sw2d_comp_wall", lambda: cases.radial_dam(n=38, char_decomp=0, tfluct_solver=0, mthbc=(3, 3, 1, 1))),
    ("acoustics2d_cd2", lambda: cases.acoustics2d(n=41, char_decomp=2)),
]


def _run(ps, q, aux, precision, variant):
    with S.Solver(ps, precision) as s:
        s.select_tiles(variant)
        s.set_aux(aux) if aux is not None else None
        s.set_q(q)
        res = s.sharpclaw(0.0, RUN["tend"], RUN["dt_initial"], RUN["cfl_max"], RUN["cfl_desired"])
        tiles = s.tiles()
        return s.get_q(), res, tiles


TOL = {"fp64_strict": 0.0, "fp64": 1e-13, "mixed": 1e-6}


def _same(a, b, precision):
    if precision == "fp64_strict":
        return np.array_equal(a, b)
    err = max(np.abs(a[m] - b[m]).max() / max(np.abs(b[m]).max(), 1e-300) for m in range(a.shape[0]))
    return err <= TOL[precision]


@pytest.mark.parametrize("name,make", TILE_CASES, ids=[c[0] for c in TILE_CASES])
@pytest.mark.parametrize("precision", ["fp64_strict", "fp64", "mixed"])
def test_tile_shapes_agree(name, make, precision):
    po, ps, q, aux = make()
    q0, r0, t0 = _run(ps, q, aux, precision, 0)
    assert t0["variant"] == 0 and not t0["tuned"]
    assert r0["info"] == 0 and r0["steps_taken"] > 3
    for v in range(1, len(S.Solver.TILE_SHAPES)):
        qv, rv, tv = _run(ps, q, aux, precision, v)
        assert tv["variant"] == v
        assert rv["steps_taken"] == r0["steps_taken"]
        assert _same(qv, q0, precision), f"shape {v} differs"
        if precision == "fp64_strict":
            assert rv["cfl_maxused"] == r0["cfl_maxused"]
    qa, ra, ta = _run(ps, q, aux, precision, -1)
    assert ta["tuned"] and all(ms > 0 for ms in ta["trial_ms"])
    # the fastest shape, or shape 0 when none beats it by more than 2%
    ms = ta["trial_ms"]
    best = int(np.argmin(ms))
    assert ta["variant"] == (best if ms[best] < 0.98 * ms[0] else 0)
    assert _same(qa, q0, precision) and ra["steps_taken"] == r0["steps_taken"]
    if precision == "fp64_strict":
        qo, ro = O.sharpclaw(po, q, aux, tstart=0.0, time_integrator=3, **RUN)
        assert ro.steps_taken == r0["steps_taken"]
        assert np.array_equal(q0[:, 3:-3, 3:-3], qo[:, 3:-3, 3:-3])


def test_select_tiles_rejects():
    _, ps, q, _ = cases.radial_dam(n=16)
    with S.Solver(ps, "fp64") as s:
        with pytest.raises(Exception):
            s.select_tiles(len(S.Solver.TILE_SHAPES))
    _, ps1, _, _ = cases.shu_osher(mx=64)
    with S.Solver(ps1, "fp64") as s:
        s.select_tiles(0)
        s.select_tiles(-1)
        with pytest.raises(Exception):
            s.select_tiles(1)
        assert s.tiles()["variant"] == 0
