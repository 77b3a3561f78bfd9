"""The allocation-free SSP-RK step, scl_rk_step_noalloc, on a GPU.

Some callers of this library cannot allocate device memory while they run: a
host time loop that calls the step once per time step from code that must not
synchronise the device (cudaMalloc/cudaFree may stall all streams), or a host
that hands every library a fixed memory budget at start-up and forbids later
allocations.  scl_rk_step_noalloc takes the caller's device arrays and keeps
its Runge-Kutta stage registers in a fixed device array inside the library.

Through the C ABI, these tests check that two calls in a row give the same
states and CFL numbers as two calls of the existing handle-based step
(scl_rk_step), bit for bit in FP64_STRICT and within the 1e-12 relative bound
of the other FP64 parity tests otherwise (walls and the mixed-form paired
kernel included, on caller planes of even and odd length); that two calls
equal two steps of the oracle bit for bit; that repeated calls allocate no
device memory; that a grid larger than the fixed scratch is rejected; and
that a host array is refused before anything is launched.
The file is collected last so that a failure here never hides another test.
"""
import ctypes

import numpy as np
import pytest

import cases
import sharpclaw_b200 as S
from sharpclaw_b200 import _capi as C

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12

CASES = [
    ("euler_ssp104_strict", "fp64_strict", lambda: cases.shu_osher(mx=777), 4),
    ("euler_ssp33_fp64", "fp64", lambda: cases.shu_osher(mx=500, char_decomp=0), 3),
    ("acoustics_ssp104_mixed", "mixed", lambda: cases.acoustics1d(mx=400), 4),
    ("advection_ssp22_strict", "fp64_strict", lambda: cases.advection(mx=300), 1),
    ("advection_ssp42_strict", "fp64_strict", lambda: cases.advection(mx=129, mthbc=(1, 1)), 2),
    # solid walls on both sides (bc1.f90 mthbc = 3: mirror, momentum negated)
    ("euler_wall_ssp33_strict", "fp64_strict", lambda: cases.shu_osher(mx=300, mthbc=(3, 3), perturb=0.05), 3),
    ("acoustics_wall_ssp104_strict", "fp64_strict", lambda: cases.acoustics1d(mx=256, mthbc=(3, 3)), 4),
    # 1-D Euler in the mixed form: the paired stage kernel on caller memory
    ("euler_ssp104_mixed", "mixed", lambda: cases.shu_osher(mx=1200), 4),
    ("euler_ssp33_mixed_odd_plane", "mixed", lambda: cases.shu_osher(mx=601, char_decomp=0), 3),
]


def _noalloc_step(cp, qd, ad, dt, stream):
    cfl = ctypes.c_double(0.0)
    rc = C.lib().scl_rk_step_noalloc(ctypes.byref(cp), ctypes.c_void_p(qd.data_ptr()),
                                     ctypes.c_void_p(ad.data_ptr() if ad is not None else 0),
                                     dt, ctypes.byref(cfl), ctypes.c_void_p(stream))
    assert rc == C.SCL_OK, C.lib().scl_last_error().decode()
    return cfl.value


@pytest.mark.parametrize("name,precision,make,ti", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_handle_step(name, precision, make, ti):
    import torch
    from oracle import oracle as O
    po, ps, q, aux = make()
    ps.time_integrator = ti
    _, _, c1 = O.step(po, q, aux, 1.0)
    dt = 0.4 / c1
    # the existing entry point, two steps in a row
    with S.Solver(ps, precision) as s:
        if aux is not None:
            s.set_aux(aux)
        s.set_q(q)
        ref_cfl = [s.rk_step(dt), s.rk_step(dt)]
        ref = s.get_q()
    # the allocation-free entry point on caller-owned device memory, two calls
    qd = torch.from_numpy(q.copy()).cuda()
    ad = torch.from_numpy(np.ascontiguousarray(aux)).cuda() if aux is not None else None
    cp = ps.to_c(C.PRECISIONS[precision])
    stream = torch.cuda.current_stream().cuda_stream
    got_cfl = [_noalloc_step(cp, qd, ad, dt, stream), _noalloc_step(cp, qd, ad, dt, stream)]
    got = qd.cpu().numpy()
    if precision == "fp64_strict":
        assert np.array_equal(got[:, 3:-3], ref[:, 3:-3])
        assert got_cfl == ref_cfl
    else:
        scale = np.abs(ref[:, 3:-3]).max()
        assert np.abs(got[:, 3:-3] - ref[:, 3:-3]).max() <= TOL_FP64 * scale
        for a, b in zip(got_cfl, ref_cfl):
            assert abs(a - b) <= TOL_FP64 * b


def test_noalloc_allocates_nothing_and_rejects_large_grids():
    import torch
    po, ps, q, aux = cases.shu_osher(mx=4000)
    ps.time_integrator = 3
    cp = ps.to_c(C.FP64)
    qd = torch.from_numpy(q.copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    _noalloc_step(cp, qd, None, 1e-4, stream)            # first call on this device
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        _noalloc_step(cp, qd, None, 1e-4, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # meqn*(mx+2*mbc) = 3*(65531+6) > 196608: refused before any launch
    big = S.ClawParams(rp=S.RP_EULER, mx=65531, dx=1e-4, mthbc=(1, 1), char_decomp=2,
                       tfluct_solver=0, time_integrator=3).to_c(C.FP64)
    cfl = ctypes.c_double(0.0)
    rc = C.lib().scl_rk_step_noalloc(ctypes.byref(big), ctypes.c_void_p(qd.data_ptr()), None, 1e-4,
                                     ctypes.byref(cfl), ctypes.c_void_p(stream))
    assert rc == C.SCL_E_INVALID
    assert b"too large" in C.lib().scl_last_error()


def test_noalloc_equals_the_oracle_directly():
    """Two allocation-free steps against two steps of the oracle (the C
    restatement of ts_ssp104), bit for bit in FP64_STRICT."""
    import torch
    from oracle import oracle as O
    po, ps, q, aux = cases.shu_osher(mx=500)
    ps.time_integrator = 4
    _, _, c1 = O.step(po, q, aux, 1.0)
    dt = 0.8 / c1
    ref, cref1 = O.rk_step(po, 4, O.bc(po, q), aux, dt)
    ref, cref2 = O.rk_step(po, 4, O.bc(po, ref), aux, dt)
    qd = torch.from_numpy(q.copy()).cuda()
    cp = ps.to_c(C.FP64_STRICT)
    stream = torch.cuda.current_stream().cuda_stream
    got_cfl = [_noalloc_step(cp, qd, None, dt, stream), _noalloc_step(cp, qd, None, dt, stream)]
    got = qd.cpu().numpy()
    assert np.array_equal(got[:, 3:-3], ref[:, 3:-3])
    assert got_cfl == [cref1, cref2]


def test_noalloc_refuses_host_memory():
    """A host array (the caller forgot to copy it to the device) is refused
    with SCL_E_INVALID before any launch; the array is left untouched."""
    import torch
    po, ps, q, aux = cases.shu_osher(mx=200)
    ps.time_integrator = 3
    cp = ps.to_c(C.FP64)
    qh = q.copy()
    cfl = ctypes.c_double(0.0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = C.lib().scl_rk_step_noalloc(ctypes.byref(cp), ctypes.c_void_p(qh.ctypes.data), None, 1e-4,
                                     ctypes.byref(cfl), ctypes.c_void_p(stream))
    assert rc == C.SCL_E_INVALID
    assert b"q_dev" in C.lib().scl_last_error()
    assert np.array_equal(qh, q)
    pinned = torch.from_numpy(q.copy()).pin_memory()
    rc = C.lib().scl_rk_step_noalloc(ctypes.byref(cp), ctypes.c_void_p(pinned.data_ptr()), None, 1e-4,
                                     ctypes.byref(cfl), ctypes.c_void_p(stream))
    assert rc == C.SCL_E_INVALID
    torch.cuda.synchronize()
