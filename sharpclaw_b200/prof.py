"""Stage-kernel probe for profilers and roofline checks.

Runs one warm-up pass plus `--reps` passes of a workload's fused stage
kernels on the device-resident state (no controller, state not advanced) and
prints the average launch time.  Used under ncu, e.g.

  python -m sharpclaw_b200.prof --workload euler1d --mx 8388608 --precision mixed --reps 1

(the warm-up pass is the first `stages` launches: skip them with `ncu -s`).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import sharpclaw_b200 as S


def euler1d(mx):
    """Shu-Osher data on [-5,5] (apps/euler/shockentropy/qinit.f:299-323)."""
    dx = 10.0 / mx
    xc = -5.0 + (np.arange(1, mx + 1) - 0.5) * dx
    q = np.zeros((3, mx + 6))
    left = xc < -4.0
    q[0, 3:-3] = np.where(left, 3.857143, 1.0 + 0.2 * np.sin(5.0 * xc))
    q[1, 3:-3] = np.where(left, 3.857143 * 2.629369, 0.0)
    q[2, 3:-3] = np.where(left, 10.333333 / 0.4 + 0.5 * 3.857143 * 2.629369 ** 2, 2.5)
    p = S.ClawParams(rp=S.RP_EULER, mx=mx, dx=dx, xlower=-5.0, mthbc=(1, 1), char_decomp=2,
                     tfluct_solver=0, time_integrator=4)
    return p, q, None, 4.5e-6 * (2 ** 20 / mx)


def sw2d(n):
    """Radial dam break on [-2.5,2.5]^2, periodic, g = 1."""
    d = 5.0 / n
    xc = -2.5 + (np.arange(n) + 0.5) * d
    X, Y = np.meshgrid(xc, xc, indexing="xy")
    q = np.zeros((3, n + 6, n + 6))
    q[0, 3:-3, 3:-3] = np.where(X ** 2 + Y ** 2 < 0.25, 2.0, 1.0)
    p = S.ClawParams(rp=S.RP_SW2D, mx=n, my=n, dx=d, dy=d, xlower=-2.5, ylower=-2.5,
                     mthbc=(2, 2, 2, 2), char_decomp=2, tfluct_solver=1, time_integrator=3)
    return p, q, None, 0.4 * d


def advection1d(mx):
    """Scalar advection on [0,1], periodic, u = 1 (apps/advection/1d): the
    lightest physics -- componentwise WENO5, Godunov rp, tfluct, SSPRK(3,3)."""
    dx = 1.0 / mx
    xc = (np.arange(mx) + 0.5) * dx
    q = np.zeros((1, mx + 6))
    q[0, 3:-3] = np.exp(-200.0 * (xc - 0.3) ** 2) + ((xc > 0.6) & (xc < 0.8))
    p = S.ClawParams(rp=S.RP_ADVECTION, mx=mx, dx=dx, mthbc=(2, 2), char_decomp=0, tfluct_solver=1,
                     time_integrator=3)
    return p, q, None, 0.8 * dx


def acoustics2d(n):
    """2-D variable-coefficient acoustics on [0,1]^2, periodic: smooth
    impedance and sound-speed fields (aux = rho*c, c), a Gaussian pressure
    pulse; componentwise WENO5, rpn2 + tfluct, SSPRK(3,3)."""
    d = 1.0 / n
    xc = (np.arange(-3, n + 3) + 0.5) * d
    X, Y = np.meshgrid(xc, xc, indexing="xy")
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    c = 1.0 + 0.2 * np.cos(2 * np.pi * X)
    aux = np.ascontiguousarray(np.stack([rho * c, c]))
    q = np.zeros((3, n + 6, n + 6))
    q[0] = np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / (2 * 0.05 ** 2))
    p = S.ClawParams(rp=S.RP_ACOUSTICS2D, mx=n, my=n, dx=d, dy=d, mthbc=(2, 2, 2, 2), char_decomp=0,
                     tfluct_solver=1, time_integrator=3)
    return p, q, aux, 0.4 * d / 1.2


WORKLOADS = {"euler1d": euler1d, "sw2d": sw2d, "advection1d": advection1d, "acoustics2d": acoustics2d}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="euler1d", choices=sorted(WORKLOADS))
    ap.add_argument("--mx", type=int, default=1 << 23)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--tiles", type=int, default=0, help="2-D tile shape (Solver.TILE_SHAPES index)")
    a = ap.parse_args()
    p, q, aux, dt = WORKLOADS[a.workload](a.mx)
    with S.Solver(p, a.precision) as s:
        if aux is not None:
            s.set_aux(aux)
        s.set_q(q)
        if p.ndim == 2:
            s.select_tiles(a.tiles)
        ms, n = s.time_stages(dt, a.reps)
    print(json.dumps({"workload": a.workload, "mx": a.mx, "precision": a.precision, "tiles": a.tiles,
                      "launches": n, "avg_launch_us": 1000.0 * ms / n}))


if __name__ == "__main__":
    main()
