"""Adjoint of the WENO / Riemann / SSP-RK step behind torch.autograd.

``WaveMisfit`` maps the initial pressure p0 of a variable-coefficient
acoustics problem (2-D q = (p, u, v) or 1-D q = (p, u), velocities zero
initially, periodic) to the misfit J = 1/2 ||p(T) - p_obs||^2 after `nsteps`
fixed-dt steps of the device solver's SSP Runge-Kutta integrator.  Its backward pass is the hand-written discrete adjoint of
the library (``scl_adjoint_step``, FP64): the forward keeps a checkpoint of q
every `checkpoint_every` steps; the backward recomputes each segment from
its checkpoint and runs the adjoint steps through it in reverse, so memory is
O(nsteps / checkpoint_every + checkpoint_every) states.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi as C
from . import ClawParams, Solver


def _interior(P: ClawParams, m: int):
    """Index of component m's interior cells (three ghost cells per side)."""
    return (m,) + (slice(3, -3),) * P.ndim


def _advance(solver: Solver, q: torch.Tensor, dt: float, nsteps: int) -> None:
    """Advance the device array q (reference layout, float64) by nsteps fixed steps in place."""
    run = C.scl_run(0.0, nsteps * dt, dt, 1e99, 1e9, 0.5, nsteps + 1, 0)
    res = C.scl_result()
    torch.cuda.current_stream().synchronize()
    C.check(C.lib().scl_sharpclaw_device(solver._h, ctypes.byref(run),
                                         ctypes.cast(q.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                         ctypes.byref(res)), "scl_sharpclaw_device")
    if res.info not in (0,) or res.steps_taken != nsteps:
        raise RuntimeError(f"forward segment stopped early: {res.steps_taken} steps, info {res.info}")


def adjoint_step(solver: Solver, q: torch.Tensor, lam: torch.Tensor, dt: float) -> torch.Tensor:
    """dJ/dq^n from q^n and dJ/dq^{n+1} (device arrays, reference layout)."""
    out = torch.zeros_like(lam)
    torch.cuda.current_stream().synchronize()
    C.check(C.lib().scl_adjoint_step(solver._h, ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(lam.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), dt), "scl_adjoint_step")
    return out


class WaveMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p0, solver: Solver, dt: float, nsteps: int, p_obs, checkpoint_every: int = 20):
        P: ClawParams = solver.params
        q = torch.zeros(P.shape(), dtype=torch.float64, device=p0.device)
        q[_interior(P, 0)] = p0.detach().to(torch.float64)
        ckpts, lens = [], []
        done = 0
        while done < nsteps:
            k = min(checkpoint_every, nsteps - done)
            ckpts.append(q.clone())
            lens.append(k)
            _advance(solver, q, dt, k)
            done += k
        r = q[_interior(P, 0)] - p_obs
        ctx.solver, ctx.dt, ctx.lens = solver, dt, lens
        ctx.save_for_backward(r, *ckpts)
        return 0.5 * (r * r).sum()

    @staticmethod
    def backward(ctx, gJ):
        r, *ckpts = ctx.saved_tensors
        solver, dt = ctx.solver, ctx.dt
        lam = torch.zeros_like(ckpts[0])
        lam[_interior(solver.params, 0)] = gJ * r
        for q0, k in zip(reversed(ckpts), reversed(ctx.lens)):
            states = [q0.clone()]
            for _ in range(k - 1):                    # recompute the segment
                q = states[-1].clone()
                _advance(solver, q, dt, 1)
                states.append(q)
            for q in reversed(states):
                lam = adjoint_step(solver, q, lam, dt)
        return lam[_interior(solver.params, 0)].clone(), None, None, None, None, None


def wave_misfit(p0, solver: Solver, dt: float, nsteps: int, p_obs, checkpoint_every: int = 20):
    """J(p0) = 1/2 ||p(T) - p_obs||^2 with the library's hand-written adjoint as backward."""
    return WaveMisfit.apply(p0, solver, dt, nsteps, p_obs, checkpoint_every)
