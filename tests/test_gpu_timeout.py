"""Failure detection of the bounded waits, on a GPU, without faulting it.

The 1-D Euler stage kernels (the paired kernel of the FP32 forms and the
one-interface kernel of the FP64 forms) stage their tiles by bulk copies
completed on an mbarrier; every wait on it is bounded.
scl_test_wait_timeout makes the handle's stage launches announce 16 bytes
that no copy delivers and bounds each wait at 1 ms, so every wait runs out
(a flag nothing sets): the kernels raise SCL_STATUS_TIMEOUT and finish, the
controller discards the step, and the host gets SCL_E_TIMEOUT.  Switched off
again, the same handle steps normally and equals the oracle.
"""
import numpy as np
import pytest

import cases
from oracle import oracle as O
import sharpclaw_b200 as S
from sharpclaw_b200 import _capi as C

pytestmark = pytest.mark.gpu

CASES = [
    ("euler_paired_mixed", lambda: cases.shu_osher(mx=300), "mixed"),
    ("euler_paired_fp32", lambda: cases.shu_osher(mx=700, char_decomp=0), "fp32"),
    ("euler_one_interface_fp64_strict", lambda: cases.shu_osher(mx=300), "fp64_strict"),
    ("euler_one_interface_fp64", lambda: cases.shu_osher(mx=500), "fp64"),
]


@pytest.mark.parametrize("name,make,precision", CASES, ids=[c[0] for c in CASES])
def test_wait_timeout_is_reported_and_recovers(name, make, precision):
    po, ps, q, aux = make()
    ps.time_integrator = 3
    _, _, c1 = O.step(po, q, aux, 1.0)
    dt = 0.4 / c1
    with S.Solver(ps, precision) as s:
        s.set_q(q)
        q_before = s.get_q()
        assert C.lib().scl_test_wait_timeout(s._h, 1) == C.SCL_OK
        with pytest.raises(S.SharpClawError) as e:
            s.rk_step(dt)
        assert e.value.code == C.SCL_E_TIMEOUT
        # the time loop in step graphs (a small grid's cluster-resident loop
        # stages by the threads and has no such waits): the first step is
        # discarded and the run stops
        s.set_run_mode(S.RUN_GRAPH)
        run = s._run(0.0, 10 * dt, dt, 1e99, 1e9, 0.5, 100, 1)
        res = C.scl_result()
        rc = C.lib().scl_sharpclaw(s._h, run, res)
        assert rc == C.SCL_E_TIMEOUT
        assert res.status & C.STATUS_TIMEOUT and res.steps_taken == 0 and res.tend == 0.0
        assert np.array_equal(s.get_q(), q_before)            # q = qold
        # normal operation again on the same handle
        assert C.lib().scl_test_wait_timeout(s._h, 0) == C.SCL_OK
        s.set_q(q)
        cfl = s.rk_step(dt)
        got = s.get_q()
    ref, cref = O.rk_step(po, 3, O.bc(po, q), aux, dt)
    sl = (slice(None), slice(3, -3)) if ps.ndim == 1 else (slice(None), slice(3, -3), slice(3, -3))
    if precision == "fp64_strict":
        assert np.array_equal(got[sl], ref[sl]) and cfl == cref
    else:
        assert np.abs(got[sl] - ref[sl]).sum() <= 1e-5 * np.abs(ref[sl]).sum()
