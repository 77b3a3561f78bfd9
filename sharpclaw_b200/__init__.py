"""sharpclaw_b200 -- SharpClaw's semi-discrete WENO step on NVIDIA B200 (sm_100a).

Host-side mirror of the reference's operator interface for the hot path:

===========================  ==============================================
reference (Fortran)          here
===========================  ==============================================
module ClawParams            :class:`ClawParams`
step (1d/step1d.f90,         :meth:`Solver.step`   -> (q with ghosts, dq, cfl)
      2d/step2d.f90)
flux1 (src/flux1.f90)        :meth:`Solver.flux1`  -> (dq1d, cfl)
ts_ssp22/42/33/104           :meth:`Solver.rk_step`
sharpclaw (src/sharpclaw.f90) :meth:`Solver.sharpclaw` / :func:`sharpclaw`
===========================  ==============================================

Arrays use the reference layout: numpy float64 arrays of shape
``(meqn, mx+2*mbc)`` (1-D) or ``(meqn, my+2*mbc, mx+2*mbc)`` (2-D), C order,
which is byte-for-byte the Fortran column-major ``q(1-mbc:mx+mbc[,1-mbc:my+mbc],meqn)``.
All compute runs in the CUDA library; a missing library is an error.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi as C
from ._capi import (B4STEP_NONE, B4STEP_SWIRL, B4STEP_TIME_REVERSAL, BC_USER_NONE, BC_USER_OSCILLATING_WALL, FP32, FP64, FP64_STRICT, MIXED,  # noqa: F401
                    RP_ACOUSTICS_CONST, RP_ACOUSTICS_FWAVE, RP_ADVECTION_CONS, RP_STEGOTON, RP_TRAFFIC,
                    RP_ACOUSTICS1D, RP_ACOUSTICS2D, RP_ADVECTION, RP_ADVECTION2D, RP_EULER, RP_SW1D, RP_SW2D,
                    RP_SWF_BATHY, RP_SWF_KAPPA, RP_SWF_RADIAL, SRC_BATHYMETRY_SW, SRC_NONE, SRC_RADIAL_SW,
                    RUN_AUTO, RUN_GRAPH, RUN_RESIDENT, SharpClawError)

from .datafile import claw_params, read_sharpclaw_data, run_settings  # noqa: E402,F401

__all__ = ["ClawParams", "Solver", "Batch", "sharpclaw", "SharpClawError", "read_sharpclaw_data",
           "claw_params", "run_settings", "RP_ADVECTION", "RP_EULER",
           "RP_SW2D", "RP_ACOUSTICS1D", "RP_ACOUSTICS2D", "RP_ADVECTION2D", "RP_SW1D", "RP_SWF_BATHY", "RP_SWF_RADIAL", "RP_SWF_KAPPA",
           "RP_ACOUSTICS_CONST", "RP_ACOUSTICS_FWAVE", "RP_TRAFFIC", "RP_ADVECTION_CONS",
           "RP_STEGOTON",
           "SRC_NONE", "SRC_RADIAL_SW",
           "SRC_BATHYMETRY_SW", "B4STEP_NONE", "B4STEP_SWIRL",
           "RUN_AUTO", "RUN_GRAPH", "RUN_RESIDENT", "BC_USER_NONE", "BC_USER_OSCILLATING_WALL",
           "B4STEP_TIME_REVERSAL"]

# plugin id -> (meqn, mwaves, maux, ndim)
PLUGINS = {
    RP_ADVECTION: (1, 1, 0, 1),
    RP_EULER: (3, 3, 0, 1),
    RP_SW2D: (3, 3, 0, 2),
    RP_ACOUSTICS1D: (2, 2, 2, 1),
    RP_ACOUSTICS2D: (3, 2, 2, 2),
    RP_ADVECTION2D: (1, 1, 2, 2),
    RP_SW1D: (2, 2, 0, 1),
    RP_SWF_BATHY: (2, 2, 1, 1),
    RP_SWF_RADIAL: (2, 2, 2, 1),
    RP_SWF_KAPPA: (2, 2, 4, 1),
    RP_ACOUSTICS_CONST: (2, 2, 0, 1),
    RP_ACOUSTICS_FWAVE: (2, 2, 2, 1),
    RP_TRAFFIC: (1, 1, 1, 1),
    RP_ADVECTION_CONS: (1, 1, 1, 1),
    RP_STEGOTON: (2, 2, 3, 1),
}


@dataclass
class ClawParams:
    """Module ClawParams (src/ClawParams.f90:1-16) plus the plugin COMMON
    blocks (/comrp/ u or g, /param/ gamma) and the integrator choice."""
    rp: int
    mx: int
    dx: float
    my: int = 1
    dy: float = 1.0
    ndim: Optional[int] = None
    meqn: Optional[int] = None
    mwaves: Optional[int] = None
    maux: Optional[int] = None
    mbc: int = 3
    mcapa: int = 0
    lim_type: int = 2
    char_decomp: int = 0
    tfluct_solver: int = 1
    mthbc: Sequence[int] = field(default_factory=lambda: (2, 2, 2, 2))
    xlower: float = 0.0
    ylower: float = 0.0
    efix: Optional[int] = None
    u: float = 1.0
    gamma: float = 1.4
    grav: float = 1.0
    time_integrator: int = 3
    mthlim: Sequence[int] = field(default_factory=lambda: (1, 1, 1, 1))
    src_term: int = 0
    rho: float = 1.0      # homogeneous acoustics (common /cparam/)
    bulk: float = 1.0
    # mthbc = 0 sides: the app's bc1.f on the device (BC_USER_OSCILLATING_WALL:
    # apps/elasticity/stegoton/bc1.f with wall = (t1, a1, tw1, t2, a2, tw2))
    bc_user: int = 0
    wall: Sequence[float] = (0.0, 0.0, 1.0, 0.0, 0.0, 1.0)

    def __post_init__(self):
        meqn, mwaves, maux, ndim = PLUGINS.get(self.rp, (None, None, 0, None))
        if self.meqn is None:
            self.meqn = meqn
        if self.mwaves is None:
            self.mwaves = mwaves
        if self.maux is None:
            self.maux = maux
        if self.ndim is None:
            self.ndim = ndim
        if self.efix is None:
            # rp1eu.f:40 and 1dRadialSymm-qwave/rp1sw.f: efix .true.; rpn2sw.f:48 .false.
            self.efix = 1 if self.rp in (RP_EULER, RP_SW1D) else 0
        if self.ndim == 1:
            self.my = 1

    def shape(self, ncomp: Optional[int] = None):
        n = self.meqn if ncomp is None else ncomp
        if self.ndim == 1:
            return (n, self.mx + 2 * self.mbc)
        return (n, self.my + 2 * self.mbc, self.mx + 2 * self.mbc)

    def to_c(self, precision: int) -> C.scl_params:
        p = C.scl_params()
        p.ndim, p.mx, p.my = self.ndim, self.mx, self.my
        p.meqn, p.mwaves, p.mbc, p.maux, p.mcapa = self.meqn, self.mwaves, self.mbc, self.maux, self.mcapa
        p.lim_type, p.char_decomp, p.tfluct_solver = self.lim_type, self.char_decomp, self.tfluct_solver
        for k in range(4):
            p.mthbc[k] = int(self.mthbc[k]) if k < len(self.mthbc) else 2
        p.dx, p.dy, p.xlower, p.ylower = self.dx, self.dy, self.xlower, self.ylower
        p.rp, p.efix = self.rp, int(self.efix)
        p.u, p.gamma, p.grav = self.u, self.gamma, self.grav
        p.time_integrator, p.precision = self.time_integrator, precision
        for k in range(4):
            p.mthlim[k] = int(self.mthlim[k]) if k < len(self.mthlim) else 1
        p.src_term = int(self.src_term)
        p.rho, p.bulk = float(self.rho), float(self.bulk)
        p.bc_user = int(self.bc_user)
        for k in range(6):
            p.wall[k] = float(self.wall[k])
        return p


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return ctypes.POINTER(ctypes.c_double)()
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("arrays must be C-contiguous float64 in the reference layout")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _precision(precision) -> int:
    if isinstance(precision, str):
        return C.PRECISIONS[precision]
    return int(precision)


class Solver:
    """One grid on the current CUDA device (a handle of the C ABI)."""

    def __init__(self, params: ClawParams, precision="fp64"):
        self.params = params
        self.precision = _precision(precision)
        self._cp = params.to_c(self.precision)
        h = ctypes.c_void_p()
        C.check(C.lib().scl_create(ctypes.byref(self._cp), ctypes.byref(h)), "scl_create")
        self._h = h

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            C.lib().scl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ------------------------------------------------------------------
    def _check_field(self, a, ncomp=None):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.params.shape(ncomp):
            raise ValueError(f"expected shape {self.params.shape(ncomp)}, got {a.shape}")
        return a

    def set_q(self, q):
        q = self._check_field(q)
        C.check(C.lib().scl_set_q(self._h, _ptr(q)), "scl_set_q")

    def get_q(self) -> np.ndarray:
        q = np.empty(self.params.shape(), dtype=np.float64)
        C.check(C.lib().scl_get_q(self._h, _ptr(q)), "scl_get_q")
        return q

    def set_aux(self, aux):
        if self.params.maux == 0:
            return
        aux = self._check_field(aux, self.params.maux)
        C.check(C.lib().scl_set_aux(self._h, _ptr(aux)), "scl_set_aux")

    # -- operators ----------------------------------------------------------------
    def step(self, q, dt: float, t: float = 0.0):
        """step1d/step2d: bc + src + flux1/flux2.  Returns (q with ghost cells
        filled, dq = dt*L(q) on interior cells, cfl)."""
        q = self._check_field(q).copy()
        dq = np.zeros_like(q)
        cfl = ctypes.c_double(0.0)
        C.check(C.lib().scl_step_dq(self._h, _ptr(q), _ptr(dq), dt, t, ctypes.byref(cfl)), "scl_step_dq")
        return q, dq, cfl.value

    def flux1(self, q1d, dt: float, aux1d=None, ixy: int = 1):
        """flux1.f90 on one line: q1d shape (meqn, mx+2mbc); returns (dq1d, cfl)."""
        q1d = np.ascontiguousarray(q1d, dtype=np.float64)
        meqn, ld = q1d.shape
        mx = ld - 2 * self.params.mbc
        a = None if aux1d is None else np.ascontiguousarray(aux1d, dtype=np.float64)
        dq = np.zeros_like(q1d)
        cfl = ctypes.c_double(0.0)
        C.check(C.lib().scl_flux1(self._h, _ptr(q1d), _ptr(a), _ptr(dq), dt, ixy, mx, ctypes.byref(cfl)),
                "scl_flux1")
        return dq, cfl.value

    def rk_step(self, dt: float, told: float = 0.0) -> float:
        """One SSP-RK step on the device-resident q; returns the last stage's CFL."""
        cfl = ctypes.c_double(0.0)
        C.check(C.lib().scl_rk_step(self._h, dt, told, ctypes.byref(cfl)), "scl_rk_step")
        return cfl.value

    @staticmethod
    def _run(tstart, tend, dt_initial, dt_max, cfl_max, cfl_desired, max_steps, dt_variable):
        return C.scl_run(tstart, tend, dt_initial, dt_max, cfl_max, cfl_desired, max_steps, dt_variable)

    def sharpclaw(self, tstart: float, tend: float, dt_initial: float, cfl_max: float,
                  cfl_desired: float, dt_max: float = 1e99, max_steps: int = 50000,
                  dt_variable: int = 1) -> dict:
        """The time loop of sharpclaw() on the device; returns its outputs."""
        run = self._run(tstart, tend, dt_initial, dt_max, cfl_max, cfl_desired, max_steps, dt_variable)
        res = C.scl_result()
        rc = C.lib().scl_sharpclaw(self._h, ctypes.byref(run), ctypes.byref(res))
        if rc not in (C.SCL_OK, C.SCL_E_NONFINITE):
            C.check(rc, "scl_sharpclaw")
        return {k: getattr(res, k) for k, _ in C.scl_result._fields_}

    def time_steps(self, nsteps: int, dt_initial: float, cfl_max: float, cfl_desired: float,
                   tend: float = 1e30, dt_variable: int = 1):
        """Run exactly `nsteps` controller steps from the device-resident state and
        return (elapsed device ms, result dict)."""
        run = self._run(0.0, tend, dt_initial, 1e99, cfl_max, cfl_desired, nsteps, dt_variable)
        res = C.scl_result()
        ms = ctypes.c_float(0.0)
        C.check(C.lib().scl_time_steps(self._h, ctypes.byref(run), nsteps, ctypes.byref(ms),
                                       ctypes.byref(res)), "scl_time_steps")
        return ms.value, {k: getattr(res, k) for k, _ in C.scl_result._fields_}


    def time_stages(self, dt: float, reps: int):
        """Time `reps` passes of the stage kernels (no controller, state not
        advanced); returns (elapsed device ms, number of kernel launches)."""
        ms = ctypes.c_float(0.0)
        n = ctypes.c_longlong(0)
        C.check(C.lib().scl_time_stages(self._h, dt, reps, ctypes.byref(ms), ctypes.byref(n)),
                "scl_time_stages")
        return ms.value, n.value

    @property
    def kernels_per_step(self) -> int:
        return C.lib().scl_kernels_per_step(self._h)

    def set_run_mode(self, mode: int):
        """RUN_GRAPH: step graphs; RUN_RESIDENT: the whole controller loop in
        one thread-block cluster (1-D grids of at most 8128 cells); RUN_AUTO
        (default): resident up to 1016 cells."""
        C.check(C.lib().scl_set_run_mode(self._h, int(mode)), "scl_set_run_mode")

    def set_totals(self, on: bool = True):
        """Keep the conserved totals sum(q [* kappa]) * dx [* dy] of every
        component in FP64 with compensated summation, at the start of each
        sharpclaw() / time_steps() run and after every accepted step (one
        kernel per step in graph runs; summed by the tile code in
        cluster-resident runs)."""
        C.check(C.lib().scl_set_totals(self._h, int(bool(on))), "scl_set_totals")

    def conserved_totals(self):
        """dict(tot0, tot, drift) of the last run: the totals at its start, of
        the current state, and the largest |tot - tot0| over its accepted
        steps (numpy arrays of meqn values)."""
        m = self.params.meqn
        a, b, c = (np.zeros(m) for _ in range(3))
        C.check(C.lib().scl_conserved_totals(self._h, _ptr(a), _ptr(b), _ptr(c)), "scl_conserved_totals")
        return {"tot0": a, "tot": b, "drift": c}

    def last_run(self):
        """(mode, kernel launches) of the last sharpclaw() / time_steps()."""
        m, n = ctypes.c_int(), ctypes.c_longlong()
        C.check(C.lib().scl_last_run(self._h, ctypes.byref(m), ctypes.byref(n)), "scl_last_run")
        return m.value, n.value

    def write_frame(self, t: float, iframe: int, dir: str | None = None, write_aux: bool | None = None):
        """Write fort.qNNNN / fort.tNNNN (/ fort.aNNNN) of the current state in
        the format of out1.f90 / out2.f90 without stalling the device; the
        files are complete after wait_frames() (or the next write_frame).
        write_aux defaults to the reference's choice: 1-D no, 2-D yes."""
        if write_aux is None:
            write_aux = self.params.ndim == 2
        d = None if dir is None else os.fsencode(dir)
        C.check(C.lib().scl_write_frame(self._h, float(t), int(iframe), d, int(bool(write_aux))),
                "scl_write_frame")

    def set_b4step(self, kind: int, param: float = 0.0):
        """Run a b4step hook on the device before every new time step of
        sharpclaw() (B4STEP_SWIRL: param = tperiod, and the aux set with
        set_aux is the hook's base field; B4STEP_TIME_REVERSAL: param =
        trtime, apps/elasticity/stegoton/b4step1.f)."""
        C.check(C.lib().scl_set_b4step(self._h, int(kind), float(param)), "scl_set_b4step")

    def wait_frames(self):
        C.check(C.lib().scl_wait_frames(self._h), "scl_wait_frames")

    def run_frames(self, t0: float, dt_initial: float, cfl_max: float, cfl_desired: float, *,
                   nout: int = 0, tfinal: float | None = None, tout=None, outdir: str | None = None,
                   dt_max: float = 1e99, max_steps: int = 50000, dt_variable: int = 1,
                   write_aux: bool | None = None) -> list:
        """The output loop of src/main.f90:170-245 on the device-resident
        state: frame 0 at t0, then for each output time a sharpclaw() call
        from the previous one (outstyle 1: nout equal intervals to tfinal;
        outstyle 2: the times in tout), dt_initial carried over as the last
        dt (main.f90:220), and frame n written from the device without
        stalling it.  Returns the result dict of every interval; a non-zero
        info is returned, not raised, as main.f90 reports it and goes on."""
        if tout is None:
            if nout < 1 or tfinal is None:
                raise ValueError("give nout and tfinal (outstyle 1) or tout (outstyle 2)")
            dtout = (tfinal - t0) / nout
            times = None
        else:
            times = [float(x) for x in tout]
            nout = len(times)
        self.write_frame(t0, 0, outdir, write_aux)
        results = []
        tend = t0
        dt = dt_initial
        for n in range(1, nout + 1):
            tstart = tend
            tend = tstart + dtout if times is None else times[n - 1]        # main.f90:180-186
            res = self.sharpclaw(tstart, tend, dt, cfl_max, cfl_desired, dt_max=dt_max, max_steps=max_steps,
                                 dt_variable=dt_variable)
            results.append(res)
            dt = res["dt_last"]                                              # :220
            self.write_frame(tend, n, outdir, write_aux)                     # :230-233
        self.wait_frames()
        return results

    TILE_SHAPES = ((16, 7, 128), (32, 7, 256), (16, 15, 256))  # (cells x, cells y, threads)

    def select_tiles(self, variant: int = -1):
        """Fix the 2-D stage kernel's tile shape (index into TILE_SHAPES), or
        with -1 let the next run time every shape and keep the fastest."""
        C.check(C.lib().scl_select_tiles(self._h, int(variant)), "scl_select_tiles")

    def tiles(self):
        """Shape in use, whether it was chosen by timing, per-shape trial ms."""
        v, t = ctypes.c_int(), ctypes.c_int()
        tm = (ctypes.c_float * len(self.TILE_SHAPES))()
        C.check(C.lib().scl_tiles(self._h, ctypes.byref(v), ctypes.byref(t), tm), "scl_tiles")
        return {"variant": v.value, "shape": self.TILE_SHAPES[v.value], "tuned": bool(t.value),
                "trial_ms": list(tm)}


def sharpclaw(params: ClawParams, q, aux=None, *, tstart: float, tend: float, dt_initial: float,
              cfl_max: float, cfl_desired: float, dt_max: float = 1e99, max_steps: int = 50000,
              dt_variable: int = 1, precision="fp64"):
    """Functional form of sharpclaw(): returns (q at the final time, outputs)."""
    with Solver(params, precision) as s:
        s.set_aux(aux) if aux is not None else None
        s.set_q(q)
        res = s.sharpclaw(tstart, tend, dt_initial, cfl_max, cfl_desired, dt_max, max_steps, dt_variable)
        return s.get_q(), res


def write_frame(params: ClawParams, q, aux=None, *, t: float, iframe: int, dir: str | None = None,
                write_aux: bool | None = None):
    """Frame files of out1.f90 / out2.f90 from host arrays (no GPU needed)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    if q.shape != params.shape():
        raise ValueError(f"q has shape {q.shape}, expected {params.shape()}")
    if write_aux is None:
        write_aux = params.ndim == 2
    a = None
    if write_aux and params.maux > 0:
        if aux is None:
            raise ValueError("write_aux needs aux")
        a = np.ascontiguousarray(aux, dtype=np.float64)
    cp = params.to_c(FP64)
    d = None if dir is None else os.fsencode(dir)
    C.check(C.lib().scl_format_frame(ctypes.byref(cp), _ptr(q), _ptr(a), float(t), int(iframe), d,
                                     int(bool(write_aux))), "scl_format_frame")


class Batch:
    """Many independent 1-D problems of uneven size, each with its own
    sharpclaw() controller, advanced together (batched persistent launches).

    ``params`` gives the plugin, options, integrator (its mx/dx are ignored);
    ``mx`` and ``dx`` give every instance's cells and spacing.  State arrays
    are the instances' reference-layout arrays concatenated."""

    def __init__(self, params: ClawParams, mx, dx, precision="fp32"):
        self.params = params
        self.mx = np.ascontiguousarray(mx, dtype=np.int32)
        self.dx = np.ascontiguousarray(dx, dtype=np.float64)
        self.ninst = len(self.mx)
        self.precision = _precision(precision)
        self._cp = params.to_c(self.precision)
        h = ctypes.c_void_p()
        C.check(C.lib().scl_batch_create(ctypes.byref(self._cp), self.ninst, self.mx.ctypes.data,
                                         self.dx.ctypes.data, ctypes.byref(h)), "scl_batch_create")
        self._h = h
        ld = self.mx.astype(np.int64) + 2 * params.mbc
        self.offsets = np.concatenate([[0], np.cumsum(ld * params.meqn)])

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            C.lib().scl_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def pack(self, qs):
        """Concatenate per-instance arrays of shape (meqn, mx[k]+6)."""
        return np.ascontiguousarray(np.concatenate([np.ascontiguousarray(q, np.float64).ravel() for q in qs]))

    def unpack(self, flat, ncomp=None):
        n = self.params.meqn if ncomp is None else ncomp
        out, o = [], 0
        for m in self.mx:
            size = n * (int(m) + 2 * self.params.mbc)
            out.append(flat[o:o + size].reshape(n, int(m) + 2 * self.params.mbc))
            o += size
        return out

    def set_q(self, qs):
        flat = self.pack(qs)
        C.check(C.lib().scl_batch_set_q(self._h, _ptr(flat)), "scl_batch_set_q")

    def get_q(self):
        flat = np.empty(int(self.offsets[-1]), dtype=np.float64)
        C.check(C.lib().scl_batch_get_q(self._h, _ptr(flat)), "scl_batch_get_q")
        return self.unpack(flat)

    def set_aux(self, auxs):
        flat = self.pack(auxs)
        C.check(C.lib().scl_batch_set_aux(self._h, _ptr(flat)), "scl_batch_set_aux")

    def sharpclaw(self, tstart, tend, dt_initial, cfl_max, cfl_desired, dt_max=1e99, max_steps=50000,
                  dt_variable=1):
        """sharpclaw() on every instance; dt_initial is a scalar or one value
        per instance.  Returns (list of per-instance output dicts, device ms)."""
        run = C.scl_run(tstart, tend, float(np.max(dt_initial)), dt_max, cfl_max, cfl_desired, max_steps,
                        dt_variable)
        dt0 = np.ascontiguousarray(np.broadcast_to(np.asarray(dt_initial, np.float64), (self.ninst,)))
        res = (C.scl_result * self.ninst)()
        ms = ctypes.c_float(0.0)
        C.check(C.lib().scl_batch_run(self._h, ctypes.byref(run), dt0.ctypes.data, ctypes.addressof(res),
                                      ctypes.byref(ms)), "scl_batch_run")
        out = [{k: getattr(r, k) for k, _ in C.scl_result._fields_} for r in res]
        return out, ms.value

    def select(self, variant: int = -1):
        """Fix the tile variant (0, 1) or let the next run choose (-1)."""
        C.check(C.lib().scl_batch_select(self._h, int(variant)), "scl_batch_select")

    def launches(self) -> int:
        """Kernel launches of the last sharpclaw() call."""
        return int(C.lib().scl_batch_launches(self._h))

    def tuning(self):
        v, nt, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        tm = (ctypes.c_float * 3)()
        C.check(C.lib().scl_batch_tuning(self._h, ctypes.byref(v), ctypes.byref(nt), ctypes.byref(g), tm),
                "scl_batch_tuning")
        return {"variant": v.value, "threads": nt.value, "grid": g.value, "trial_ms": list(tm)}
