"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is the checker: tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py use it; the product
(``sharpclaw_b200``) never imports it.

Arrays use the reference's Fortran layout.  A numpy array of shape
``(meqn, mx+2*mbc)`` (1-D) or ``(meqn, my+2*mbc, mx+2*mbc)`` (2-D) in C order
has exactly the column-major ``q(1-mbc:mx+mbc[,1-mbc:my+mbc],meqn)`` memory
layout of src/1d/qalloc1.f90 / src/2d/qalloc2.f90.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libsclaw_oracle.so")

RP_ADVECTION, RP_EULER, RP_SW2D, RP_ACOUSTICS1D, RP_ACOUSTICS2D, RP_ADVECTION2D, RP_SW1D = 1, 2, 3, 4, 5, 6, 7
RP_SWF_BATHY, RP_SWF_RADIAL, RP_SWF_KAPPA = 8, 9, 10
RP_ACOUSTICS_CONST, RP_ACOUSTICS_FWAVE = 11, 12
RP_TRAFFIC, RP_ADVECTION_CONS, RP_STEGOTON = 13, 14, 15
SRC_NONE, SRC_RADIAL_SW, SRC_BATHYMETRY_SW = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("mx", ctypes.c_int), ("my", ctypes.c_int),
        ("meqn", ctypes.c_int), ("mwaves", ctypes.c_int), ("mbc", ctypes.c_int),
        ("maux", ctypes.c_int), ("mcapa", ctypes.c_int),
        ("lim_type", ctypes.c_int), ("char_decomp", ctypes.c_int),
        ("tfluct_solver", ctypes.c_int), ("mthbc", ctypes.c_int * 4),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("xlower", ctypes.c_double), ("ylower", ctypes.c_double),
        ("rp", ctypes.c_int), ("efix", ctypes.c_int),
        ("u", ctypes.c_double), ("gamma", ctypes.c_double), ("grav", ctypes.c_double),
        ("mthlim", ctypes.c_int * 4),
        ("b4step", ctypes.c_int), ("tperiod", ctypes.c_double),
        ("src_term", ctypes.c_int),
        ("rho", ctypes.c_double), ("bulk", ctypes.c_double),
        ("bc_user", ctypes.c_int), ("wall", ctypes.c_double * 6), ("bc_switched", ctypes.c_int),
        ("trtime", ctypes.c_double), ("b4_done", ctypes.c_int),
    ]


class Run(ctypes.Structure):
    _fields_ = [
        ("tstart", ctypes.c_double), ("tend", ctypes.c_double),
        ("dt_initial", ctypes.c_double), ("dt_max", ctypes.c_double),
        ("cfl_max", ctypes.c_double), ("cfl_desired", ctypes.c_double),
        ("max_steps", ctypes.c_int), ("dt_variable", ctypes.c_int),
        ("time_integrator", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("tend", ctypes.c_double), ("cfl_maxused", ctypes.c_double),
        ("cfl_last", ctypes.c_double), ("dt_minused", ctypes.c_double),
        ("dt_maxused", ctypes.c_double), ("dt_last", ctypes.c_double),
        ("steps_taken", ctypes.c_int), ("info", ctypes.c_int), ("rejected", ctypes.c_int),
        ("bc_switched", ctypes.c_int),
    ]


def build() -> str:
    """Compile the oracle with its Makefile if the library is missing or stale."""
    src = os.path.join(_HERE, "sclaw_oracle.c")
    if (not os.path.exists(_LIB)) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        dp = ctypes.POINTER(ctypes.c_double)
        P = ctypes.POINTER(Params)
        _lib.ocl_bc.argtypes = [P, dp]
        _lib.ocl_weno5.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
        _lib.ocl_weno5_char.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp]
        _lib.ocl_flux1.argtypes = [P, dp, dp, dp, ctypes.c_double, dp, ctypes.c_int, ctypes.c_int]
        _lib.ocl_step.argtypes = [P, dp, dp, dp, ctypes.c_double, ctypes.c_double, dp]
        _lib.ocl_rk_step.argtypes = [P, ctypes.c_int, dp, dp, dp, ctypes.c_double,
                                     ctypes.c_double, dp]
        _lib.ocl_sharpclaw.argtypes = [P, ctypes.POINTER(Run), dp, dp, ctypes.POINTER(Result)]
        _lib.ocl_rp.argtypes = [P, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp, dp, dp]
        _lib.ocl_evec.argtypes = [P, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp]
        _lib.ocl_tfluct.argtypes = [P, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp, dp]
        _lib.ocl_weno5_wave.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp, dp]
        _lib.ocl_output.argtypes = [P, dp, dp, ctypes.c_double, ctypes.c_int, ctypes.c_char_p,
                                    ctypes.c_int]
    return _lib


def _ptr(a):
    if a is None:
        return ctypes.POINTER(ctypes.c_double)()
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(*, ndim=1, mx, my=1, meqn, mwaves, mbc=3, maux=0, mcapa=0, char_decomp=0,
                tfluct_solver=1, mthbc=(2, 2, 2, 2), dx, dy=1.0, xlower=0.0, ylower=0.0,
                rp, efix=None, u=1.0, gamma=1.4, grav=1.0, lim_type=2, mthlim=(1, 1, 1, 1),
                src_term=SRC_NONE, rho=1.0, bulk=1.0, bc_user=0,
                wall=(0.0, 0.0, 1.0, 0.0, 0.0, 1.0)) -> Params:
    p = Params()
    p.ndim, p.mx, p.my = ndim, mx, (my if ndim == 2 else 1)
    p.meqn, p.mwaves, p.mbc, p.maux, p.mcapa = meqn, mwaves, mbc, maux, mcapa
    p.lim_type, p.char_decomp, p.tfluct_solver = lim_type, char_decomp, tfluct_solver
    for k in range(4):
        p.mthbc[k] = int(mthbc[k]) if k < len(mthbc) else 2
    p.dx, p.dy, p.xlower, p.ylower = dx, dy, xlower, ylower
    p.rp = rp
    # rp1eu.f:40 and 1dRadialSymm-qwave/rp1sw.f data efix /.true./; rpn2sw.f:48 .false.
    p.efix = (1 if rp in (RP_EULER, RP_SW1D) else 0) if efix is None else int(efix)
    p.u, p.gamma, p.grav = u, gamma, grav
    for k in range(4):
        p.mthlim[k] = int(mthlim[k]) if k < len(mthlim) else 1
    p.src_term = int(src_term)
    p.rho, p.bulk = rho, bulk
    p.bc_user = int(bc_user)
    for k in range(6):
        p.wall[k] = float(wall[k])
    return p


def field_shape(p: Params, ncomp: int):
    if p.ndim == 1:
        return (ncomp, p.mx + 2 * p.mbc)
    return (ncomp, p.my + 2 * p.mbc, p.mx + 2 * p.mbc)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with code {rc}")


def bc(p: Params, q: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).copy()
    _check(lib().ocl_bc(ctypes.byref(p), _ptr(q)), "bc")
    return q


def step(p: Params, q, aux, dt, t=0.0):
    """step1d/step2d: returns (q with ghosts filled, dq = dt*L(q), cfl)."""
    q = np.ascontiguousarray(q, dtype=np.float64).copy()
    dq = np.zeros_like(q)
    aux = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
    cfl = ctypes.c_double(0.0)
    _check(lib().ocl_step(ctypes.byref(p), _ptr(q), _ptr(dq), _ptr(aux), dt, t,
                          ctypes.byref(cfl)), "step")
    return q, dq, cfl.value


def rk_step(p: Params, time_integrator, q, aux, dt, told=0.0):
    """One SSP-RK step with qold = q; returns (q_new, cfl of the last stage)."""
    q = np.ascontiguousarray(q, dtype=np.float64).copy()
    qold = q.copy()
    aux = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
    cfl = ctypes.c_double(0.0)
    _check(lib().ocl_rk_step(ctypes.byref(p), time_integrator, _ptr(q), _ptr(qold), _ptr(aux),
                             dt, told, ctypes.byref(cfl)), "rk_step")
    return q, cfl.value


def sharpclaw(p: Params, q, aux, *, tstart, tend, dt_initial, dt_max=1e99, cfl_max, cfl_desired,
              max_steps=50000, dt_variable=1, time_integrator=3):
    q = np.ascontiguousarray(q, dtype=np.float64).copy()
    aux = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
    run = Run(tstart, tend, dt_initial, dt_max, cfl_max, cfl_desired, max_steps, dt_variable,
              time_integrator)
    res = Result()
    _check(lib().ocl_sharpclaw(ctypes.byref(p), ctypes.byref(run), _ptr(q), _ptr(aux),
                               ctypes.byref(res)), "sharpclaw")
    return q, res


def weno5(q: np.ndarray):
    """reconstruct.f90 weno5 on one line; q shape (meqn, mx2)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    meqn, mx2 = q.shape
    ql = np.zeros_like(q)
    qr = np.zeros_like(q)
    _check(lib().ocl_weno5(mx2, meqn, _ptr(q), _ptr(ql), _ptr(qr)), "weno5")
    return ql, qr


def weno5_wave(q: np.ndarray, wave: np.ndarray):
    """reconstruct.f90 weno5_wave on one line; q shape (meqn, mx2), wave shape
    (mwaves, meqn, mx2) as returned by rp() on the cell averages."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    wave = np.ascontiguousarray(wave, dtype=np.float64)
    meqn, mx2 = q.shape
    ql = np.zeros_like(q)
    qr = np.zeros_like(q)
    _check(lib().ocl_weno5_wave(mx2, meqn, wave.shape[0], _ptr(q), _ptr(wave), _ptr(ql), _ptr(qr)),
           "weno5_wave")
    return ql, qr


def evec(p: Params, q: np.ndarray, aux=None, ixy=1):
    """Plugin evec on one line; returns (evl, evr) shaped (meqn, meqn, mx2):
    evl[m-1, p-1, i] = evl(i,p,m) and evr[p-1, m-1, i] = evr(i,m,p)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    meqn, mx2 = q.shape
    mx = mx2 - 2 * p.mbc
    evl = np.zeros((meqn, meqn, mx2))
    evr = np.zeros((meqn, meqn, mx2))
    a = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
    _check(lib().ocl_evec(ctypes.byref(p), ixy, mx, _ptr(q), _ptr(a), _ptr(a), _ptr(evl),
                          _ptr(evr)), "evec")
    return evl, evr


def rp(p: Params, ql, qr, auxl=None, auxr=None, ixy=1):
    """Plugin rp on one line: interface i has left qr(i-1), right ql(i)."""
    ql = np.ascontiguousarray(ql, dtype=np.float64)
    qr = np.ascontiguousarray(qr, dtype=np.float64)
    meqn, mx2 = ql.shape
    mx = mx2 - 2 * p.mbc
    wave = np.zeros((p.mwaves, meqn, mx2))
    s = np.zeros((p.mwaves, mx2))
    amdq = np.zeros_like(ql)
    apdq = np.zeros_like(ql)
    al = None if auxl is None else np.ascontiguousarray(auxl, dtype=np.float64)
    ar = None if auxr is None else np.ascontiguousarray(auxr, dtype=np.float64)
    _check(lib().ocl_rp(ctypes.byref(p), ixy, mx, _ptr(ql), _ptr(qr), _ptr(al), _ptr(ar),
                        _ptr(wave), _ptr(s), _ptr(amdq), _ptr(apdq)), "rp")
    return wave, s, amdq, apdq


def output(p: Params, q, aux, t: float, iframe: int, dir: str, outaux: bool):
    """out1.f90 / out2.f90: writes fort.qNNNN, fort.tNNNN (and fort.aNNNN) in dir."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    a = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
    _check(lib().ocl_output(ctypes.byref(p), _ptr(q), _ptr(a), float(t), int(iframe), os.fsencode(dir),
                            int(bool(outaux))), "output")
