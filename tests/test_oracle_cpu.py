"""CPU tests of the oracle: known answers and invariants (no GPU).

The reference ships no golden vectors; its own known-answer test is
apps/acoustics/1d/interface/sharpclawtest.py, which compares SharpClaw cell
averages with the exact characteristic solution of actools.py in the 1-norm.
These tests do the same with the oracle (restated exact solution in
tests/golden/acoustics_exact.py) and add analytic invariants.
"""
import numpy as np
import pytest

import cases
from acoustics_exact import InterfaceProblem
from oracle import oracle as O


def _interface_error(mx, char_decomp):
    ap = InterfaceProblem(rho=(1.0, 4.0), c=(1.0, 0.5))
    po, _, q, aux = cases.acoustics1d(mx=mx, char_decomp=char_decomp)
    qf, res = O.sharpclaw(po, q, aux, tstart=0.0, tend=8.0, dt_initial=0.025, cfl_max=2.9,
                          cfl_desired=2.85, time_integrator=4)
    assert res.info == 0 and res.tend == 8.0
    pe, ue = ap.cell_averages(mx, res.tend)
    dx = 20.0 / mx
    return np.abs(pe - qf[0, 3:-3]).sum() * dx, np.abs(ue - qf[1, 3:-3]).sum() * dx


@pytest.mark.parametrize("char_decomp", [0, 2])
def test_acoustics_interface_known_answer(char_decomp):
    """sharpclawtest.py 'interface 1' (WENO5 / WENO5 Char, SSPRK(10,4), cfl
    2.85/2.9, t = 8): errors against the exact solution fall with mx."""
    e400, u400 = _interface_error(400, char_decomp)
    e800, u800 = _interface_error(800, char_decomp)
    assert e400 < 0.06 and e800 < 0.013
    assert np.log2(e400 / e800) > 2.0         # observed order of the pressure error
    assert np.log2(u400 / u800) > 2.0


def test_weno5_fifth_order_on_smooth_advection():
    errs = []
    for mx in (40, 80, 160):
        dx = 1.0 / mx
        po = O.make_params(mx=mx, meqn=1, mwaves=1, dx=dx, rp=O.RP_ADVECTION, u=1.0, mthbc=(2, 2))
        xe = dx * np.arange(mx + 1)
        q = np.zeros((1, mx + 6))
        q[0, 3:-3] = -(np.cos(2 * np.pi * xe[1:]) - np.cos(2 * np.pi * xe[:-1])) / (2 * np.pi * dx)
        qf, res = O.sharpclaw(po, q, None, tstart=0, tend=1.0, dt_initial=0.5 * dx, cfl_max=0.85,
                              cfl_desired=0.8, time_integrator=4)
        errs.append(np.abs(qf[0, 3:-3] - q[0, 3:-3]).sum() * dx)
    orders = [np.log2(errs[k] / errs[k + 1]) for k in range(2)]
    assert min(orders) > 4.5, orders


@pytest.mark.parametrize("make", [lambda: cases.advection(mx=200),
                                  lambda: cases.shu_osher(mx=200, mthbc=(2, 2)),
                                  lambda: cases.radial_dam(n=24)])
def test_conservation_periodic(make):
    po, _, q, aux = make()
    qb = O.bc(po, q)
    _, dq, _ = O.step(po, qb, aux, 1e-3)
    inner = dq[:, 3:-3] if po.ndim == 1 else dq[:, 3:-3, 3:-3]
    tot = np.abs(qb).sum()
    assert np.abs(inner.reshape(inner.shape[0], -1).sum(1)).max() <= 1e-12 * tot


def test_free_stream_preserved():
    po, _, q, aux = cases.shu_osher(mx=64, mthbc=(2, 2))
    q[0, :], q[1, :], q[2, :] = 1.3, 0.7, 2.9
    _, dq, _ = O.step(po, q, aux, 1e-3)
    assert np.abs(dq[:, 3:-3]).max() <= 1e-14


def test_radial_dam_xy_symmetry_is_exact():
    """Dimension-by-dimension flux2 on transposed data is the transpose."""
    po, _, q, aux = cases.radial_dam(n=30, noise=0.0)
    qT = np.stack([q[0].T, q[2].T, q[1].T])
    _, dq, _ = O.step(po, q, aux, 1e-2)
    _, dqT, _ = O.step(po, qT, aux, 1e-2)
    assert np.array_equal(dq[0], dqT[0].T)
    assert np.array_equal(dq[1], dqT[2].T)


@pytest.mark.parametrize("rp,meqn,ixys", [(O.RP_EULER, 3, (1,)), (O.RP_SW2D, 3, (1, 2))])
def test_eigenvector_plugins_are_inverse_pairs(rp, meqn, ixys):
    rng = np.random.default_rng(7)
    p = O.make_params(mx=10, meqn=meqn, mwaves=3, dx=0.1, rp=rp, mthbc=(1, 1), char_decomp=2)
    q = np.zeros((3, 16))
    q[0] = rng.uniform(0.5, 2.0, 16)
    q[1] = rng.uniform(-1, 1, 16) * q[0]
    q[2] = (rng.uniform(0.5, 2.0, 16) / 0.4 + 0.5 * q[1] ** 2 / q[0]) if rp == O.RP_EULER else rng.uniform(-1, 1, 16)
    for ixy in ixys:
        evl, evr = O.evec(p, q, ixy=ixy)
        for i in range(1, 16):
            L, R = evl[:, :, i].T, evr[:, :, i].T
            assert np.allclose(L @ R, np.eye(3), atol=1e-12)


def test_roe_property_euler_and_sw():
    """amdq + apdq = f(right) - f(left) for the Roe solvers (with and without
    the entropy fix): the flux-difference splitting the scheme relies on."""
    rng = np.random.default_rng(11)
    n = 20
    for rp, efix in ((O.RP_EULER, 1), (O.RP_EULER, 0), (O.RP_SW2D, 0), (O.RP_SW2D, 1)):
        p = O.make_params(mx=n - 6, meqn=3, mwaves=3, dx=0.1, rp=rp, efix=efix, mthbc=(1, 1))
        rho = rng.uniform(0.5, 2.0, n)
        u = rng.uniform(-2, 2, n)
        if rp == O.RP_EULER:
            pr = rng.uniform(0.5, 2.0, n)
            q = np.stack([rho, rho * u, pr / 0.4 + 0.5 * rho * u * u])

            def flux(s):
                r, m, e = s
                pp = 0.4 * (e - 0.5 * m * m / r)
                return np.array([m, m * m / r + pp, (e + pp) * m / r])
        else:
            v = rng.uniform(-1, 1, n)
            q = np.stack([rho, rho * u, rho * v])

            def flux(s):
                h, hu, hv = s
                return np.array([hu, hu * hu / h + 0.5 * h * h, hu * hv / h])
        # rp solves interface i with left state qr(i-1) and right state ql(i)
        ql, qr = q.copy(), q.copy()
        wave, s, am, ap = O.rp(p, ql, qr)
        for i in range(1, n):
            df = flux(ql[:, i]) - flux(qr[:, i - 1])
            assert np.allclose(am[:, i] + ap[:, i], df, rtol=1e-10, atol=1e-10)


def test_sw1d_roe_property_and_eigenvectors():
    """rp1sw.f (with and without its entropy fix): amdq + apdq = f(right) -
    f(left); the new 1-D shallow-water eigenvectors are inverse pairs."""
    rng = np.random.default_rng(13)
    n = 20
    h = rng.uniform(0.5, 2.0, n)
    hu = h * rng.uniform(-2, 2, n)
    q = np.stack([h, hu])

    def flux(s):
        return np.array([s[1], s[1] * s[1] / s[0] + 0.5 * s[0] * s[0]])
    for efix in (0, 1):
        p = O.make_params(mx=n - 6, meqn=2, mwaves=2, dx=0.1, rp=O.RP_SW1D, efix=efix, mthbc=(1, 1))
        wave, s, am, ap = O.rp(p, q.copy(), q.copy())
        for i in range(1, n):
            df = flux(q[:, i]) - flux(q[:, i - 1])
            assert np.allclose(am[:, i] + ap[:, i], df, rtol=1e-10, atol=1e-10)
    evl, evr = O.evec(p, q, ixy=1)
    for i in range(1, n):
        assert np.allclose(evl[:, :, i].T @ evr[:, :, i].T, np.eye(2), atol=1e-12)


@pytest.mark.parametrize("src", ["radial", "bathymetry"])
@pytest.mark.parametrize("tfluct_solver", [0, 1])
def test_source_term_known_answer(src, tfluct_solver):
    """On a uniform state every fluctuation is exactly zero, so the step's dq
    is the app's src1.f90 formula, evaluated here in numpy in the same order."""
    if src == "radial":
        po, _, q, aux = cases.radial_sw(mx=40, tfluct_solver=tfluct_solver)
        po.mthbc[0] = 1
    else:
        po, _, q, aux = cases.bathymetry_sw(mx=40, tfluct_solver=tfluct_solver)
    q[0, :], q[1, :] = 1.3, 0.4
    dt = 0.01
    _, dq, _ = O.step(po, q, aux, dt)
    i = np.arange(1, po.mx + 1)
    want = np.zeros((2, po.mx))
    if src == "radial":
        rad = po.xlower + (i - 0.5) * po.dx
        want[0] = -((dt * q[1, i + 2]) / rad)
        want[1] = -(((dt * (q[1, i + 2] * q[1, i + 2])) / q[0, i + 2]) / rad)
    else:
        want[1] = -((((po.grav * q[0, i + 2]) * (aux[0, i + 2] - aux[0, i + 1])) / po.dx) * dt)
    assert np.array_equal(dq[:, 3:-3], want)


def test_radial_sw_reproduces_2d_radial_dam():
    """The purpose of the 1dRadialSymm apps: with its radial source term the
    1-D q-wave solver reproduces the 2-D radial dam break (2dRadialDam, same
    data) along a ray, as do the two f-wave apps; without the source term the
    1-D (planar) dam break is ten times further off."""
    n = 100
    po, _, q, aux = cases.radial_dam(n=n, noise=0.0, char_decomp=0, tfluct_solver=1, mthbc=(1, 1, 1, 1))
    run = dict(tstart=0.0, tend=0.25, dt_initial=0.005, cfl_max=1.0, cfl_desired=0.9, time_integrator=4)
    q2, r2 = O.sharpclaw(po, q, aux, **run)
    xs = po.xlower + (np.arange(n) + 0.5) * po.dx
    j = n // 2
    h2 = q2[0, 3 + j, 3:-3]
    errs = {}
    for name, make in (("qwave_src", lambda: cases.radial_sw(mx=50)),
                       ("planar", lambda: cases.radial_sw(mx=50, src=False)),
                       ("fwave", lambda: cases.fwave_radial(mx=50)),
                       ("fwave_kappa", lambda: cases.fwave_radial(mx=50, kappa=True))):
        p1, _, q1, a1 = make()
        q1f, r1 = O.sharpclaw(p1, q1, a1, **run)
        assert r1.info == 0 and r1.tend == 0.25
        xc = (np.arange(p1.mx) + 0.5) * p1.dx
        h1 = np.interp(np.sqrt(xs ** 2 + xs[j] ** 2), xc, q1f[0, 3:-3])
        errs[name] = np.abs(h2 - h1).sum() / np.abs(h2).sum()
    assert errs["qwave_src"] < 0.005 and errs["planar"] > 0.03, errs
    # the f-wave apps carry the radial terms in their Riemann solvers instead
    assert errs["fwave"] < 0.008 and errs["fwave_kappa"] < 0.008, errs


@pytest.mark.parametrize("char_decomp", [0, 1])
def test_polynomial_reconstruction_third_order(char_decomp):
    """lim_type 0 (polyrecon.f90, order mthlim(1) = 3): the unlimited
    upwind-centred reconstruction converges at third order on smooth periodic
    advection (cell averages of sin 2 pi x, one period), in its componentwise
    and wave-based forms."""
    errs = []
    for mx in (40, 80, 160):
        po, _, q, aux = cases.advection(mx=mx, char_decomp=char_decomp)
        po.lim_type = 0
        po.mthlim[0] = 3
        dx = 1.0 / mx
        xc = (np.arange(mx) + 0.5) * dx
        q[0, 3:-3] = (np.cos(2 * np.pi * (xc - dx / 2)) - np.cos(2 * np.pi * (xc + dx / 2))) / (2 * np.pi * dx)
        qf, r = O.sharpclaw(po, q, aux, tstart=0.0, tend=1.0, dt_initial=0.4 * dx, cfl_max=0.5,
                            cfl_desired=0.4, time_integrator=3)
        assert r.info == 0
        errs.append(np.abs(qf[0, 3:-3] - q[0, 3:-3]).sum() * dx)
    orders = [np.log2(errs[k] / errs[k + 1]) for k in range(2)]
    assert min(orders) > 2.9, orders


def test_fwave_flat_bottom_equals_roe():
    """With a flat bottom the f-wave splitting of 1dPerturbSteady/rpf-wave.f90
    gives the Roe fluctuations of rp1sw.f without its entropy fix: the
    f-waves are s_k times the waves when the Roe matrix maps the jump in q to
    the jump in the flux."""
    rng = np.random.default_rng(3)
    n = 30
    h = rng.uniform(0.5, 2.0, n)
    q = np.stack([h, h * rng.uniform(-1, 1, n)])
    pf = O.make_params(mx=n - 6, meqn=2, mwaves=2, maux=1, dx=0.1, rp=O.RP_SWF_BATHY, grav=9.81, mthbc=(1, 1))
    pq = O.make_params(mx=n - 6, meqn=2, mwaves=2, dx=0.1, rp=O.RP_SW1D, grav=9.81, efix=0, mthbc=(1, 1))
    flat = np.zeros((1, n))
    _, sf, amf, apf = O.rp(pf, q.copy(), q.copy(), flat, flat)
    _, sq, amq, apq = O.rp(pq, q.copy(), q.copy())
    scale = np.abs(amq).max() + np.abs(apq).max()
    assert np.abs(sf[:, 1:] - sq[:, 1:]).max() <= 1e-14 * np.abs(sq).max()
    assert np.abs(amf[:, 1:] - amq[:, 1:]).max() <= 1e-13 * scale
    assert np.abs(apf[:, 1:] - apq[:, 1:]).max() <= 1e-13 * scale


def test_acoustics_fwave_interface_known_answer():
    """apps/acoustics/1d/fwave solves the interface problem of sharpclawtest.py
    in strain / momentum form (WENO5 char-wise, SSPRK(10,4), t = 8): the
    pressure -bulk*eps and velocity (rho u)/rho meet the same exact solution
    as the interface app, with the same error bounds."""
    from acoustics_exact import InterfaceProblem
    ap = InterfaceProblem()
    errs = []
    for mx in (400, 800):
        po, _, q, aux = cases.acoustics_fwave(mx=mx)
        qf, r = O.sharpclaw(po, q, aux, tstart=0.0, tend=8.0, dt_initial=0.025, cfl_max=2.5,
                            cfl_desired=2.45, time_integrator=4)
        assert r.info == 0 and r.tend == 8.0
        pe, ue = ap.cell_averages(mx, r.tend)
        dx = 20.0 / mx
        errs.append((np.abs(pe + aux[1, 3:-3] * qf[0, 3:-3]).sum() * dx,
                     np.abs(ue - qf[1, 3:-3] / aux[0, 3:-3]).sum() * dx))
    assert errs[0][0] < 0.06 and errs[1][0] < 0.013, errs
    assert np.log2(errs[0][0] / errs[1][0]) > 2.0 and np.log2(errs[0][1] / errs[1][1]) > 2.0


def test_acoustics_homogeneous_dalembert():
    """apps/acoustics/1d/homogeneous on a periodic domain: the Gaussian pulse
    splits into two waves moving at +-c (d'Alembert); cell averages of the
    exact solution at t = 0.5, errors falling with mx."""
    errs = []
    for mx in (100, 200):
        po, _, q, aux = cases.acoustics_const(mx=mx, mthbc=(2, 2), smooth=True)
        T = 0.5
        qf, r = O.sharpclaw(po, q, aux, tstart=0.0, tend=T, dt_initial=0.001, cfl_max=2.5, cfl_desired=2.4,
                            time_integrator=4)
        assert r.info == 0
        c = np.sqrt(po.bulk / po.rho)
        z = c * po.rho
        dx = 2.0 / mx
        xe = -1.0 + dx * np.arange(mx + 1)
        g, w = np.polynomial.legendre.leggauss(10)
        pts = 0.5 * (xe[:-1, None] + xe[1:, None]) + 0.5 * dx * g[None, :]

        def p0(x):
            y = (x + 1.0) % 2.0 - 1.0
            return np.exp(-50.0 * (y - 0.3) ** 2)
        pe = (0.5 * (p0(pts - c * T) + p0(pts + c * T)) * w).sum(1) * 0.5
        ue = ((p0(pts - c * T) - p0(pts + c * T)) / (2 * z) * w).sum(1) * 0.5
        errs.append((np.abs(pe - qf[0, 3:-3]).sum() * dx, np.abs(ue - qf[1, 3:-3]).sum() * dx))
    assert errs[1][0] < 2e-4 and errs[1][1] < 5e-5, errs
    assert np.log2(errs[0][0] / errs[1][0]) > 3.0, errs


def test_acoustics_app_eigenvectors_are_inverse_pairs():
    rng = np.random.default_rng(9)
    n = 16
    q = rng.uniform(-1, 1, (2, n))
    aux = np.stack([rng.uniform(0.5, 2, n), rng.uniform(0.5, 4, n)])
    for rp, kw in ((O.RP_ACOUSTICS_CONST, dict(rho=1.3, bulk=3.1)), (O.RP_ACOUSTICS_FWAVE, dict(maux=2))):
        p = O.make_params(mx=n - 6, meqn=2, mwaves=2, dx=0.1, rp=rp, mthbc=(1, 1), char_decomp=2, **kw)
        evl, evr = O.evec(p, q, aux if rp == O.RP_ACOUSTICS_FWAVE else None)
        for i in range(1, n):
            assert np.allclose(evl[:, :, i].T @ evr[:, :, i].T, np.eye(2), atol=1e-12)


@pytest.mark.parametrize("rho", [(0.2, 0.6), (0.8, 0.2)], ids=["shock", "transonic_rarefaction"])
def test_traffic_riemann_exact(rho):
    """apps/traffic/congTraffic's f-wave solver with a uniform speed limit 1:
    the LWR Riemann problem has a shock of speed 1 - rho_l - rho_r, or a fan
    rho = (1 - x/t)/2 through the sonic point (the solver's transonic split);
    L1 error of the cell averages at t = 0.5 halves with dx."""
    rl, rr = rho
    errs = []
    for mx in (200, 400):
        po, _, q, aux = cases.traffic(mx=mx, rho=rho, umax=(1.0, 1.0), lower=-1.0, upper=1.0)
        T = 0.5
        qf, r = O.sharpclaw(po, q, aux, tstart=0.0, tend=T, dt_initial=0.001, cfl_max=0.5, cfl_desired=0.45,
                            time_integrator=4)
        assert r.info == 0
        dx = 2.0 / mx
        xc = -1.0 + (np.arange(mx) + 0.5) * dx
        if rl < rr:
            ex = np.where(xc < (1.0 - rl - rr) * T, rl, rr)
        else:
            xi = xc / T
            ex = np.where(xi < 1 - 2 * rl, rl, np.where(xi > 1 - 2 * rr, rr, 0.5 * (1 - xi)))
        errs.append(np.abs(qf[0, 3:-3] - ex).sum() * dx)
    assert errs[0] < 2e-3 and errs[1] < 0.6 * errs[0], errs


def test_conservative_advection_uniform_velocity():
    """apps/traffic/flux-uq's solver with a uniform velocity is upwind
    advection: one period on a periodic domain returns the data to within the
    WENO5 error, and the total is conserved to rounding."""
    mx = 200
    po, _, q, aux = cases.advection_cons(mx=mx, u=(1.0, 1.0), lower=0.0, upper=1.0, mthbc=(2, 2))
    xc = (np.arange(mx) + 0.5) / mx
    q[0, 3:-3] = 1.0 + 0.5 * np.sin(2 * np.pi * xc)
    qf, r = O.sharpclaw(po, q, aux, tstart=0.0, tend=1.0, dt_initial=0.002, cfl_max=0.5, cfl_desired=0.45,
                        time_integrator=3)
    assert r.info == 0
    assert np.abs(qf[0, 3:-3] - q[0, 3:-3]).max() < 1e-6
    assert abs(qf[0, 3:-3].sum() - q[0, 3:-3].sum()) <= 1e-12 * q[0, 3:-3].sum()


def test_stegoton_small_strain_is_linear_acoustics():
    """apps/elasticity/stegoton's stress exp(K eps) - 1 linearises to K eps:
    for a strain pulse of amplitude 1e-6 one step of the stegoton solver
    equals, to the relative size of the neglected K eps^2 / 2 term, the step of
    the linear f-wave acoustics app on the same (rho, K) medium."""
    po, _, q, aux = cases.stegoton(mx=150, amp=1e-6)
    pl = O.make_params(meqn=2, mwaves=2, maux=2, rp=O.RP_ACOUSTICS_FWAVE, mx=po.mx, dx=po.dx, xlower=po.xlower,
                       mthbc=(1, 1), char_decomp=0, tfluct_solver=1)
    _, dqn, cfln = O.step(po, q, aux, 0.05)
    _, dql, cfll = O.step(pl, q, np.ascontiguousarray(aux[:2]), 0.05)
    scale = np.abs(dql[:, 3:-3]).max()
    assert scale > 0
    assert np.abs(dqn[:, 3:-3] - dql[:, 3:-3]).max() <= 1e-5 * scale
    assert abs(cfln - cfll) <= 1e-5 * cfll


# ---- user bc: apps/elasticity/stegoton/bc1.f (oscillating wall, switch to periodic) ----

def test_oscillating_wall_ghosts_known_answer():
    """bc1.f:100-106 at t: ghost cells mirror cells 1..3, with ghost momentum
    2 v rho(ibc) - q2(ibc), v = -a1 (1 + cos(pi (t - t1)/tw1)); extrapolation
    on the right (bc1.f:210-215)."""
    po, _, q, aux = cases.stegoton_wall(mx=48, wall=(1.0, 0.1, 1.0, 0.0, 0.0, 1.0))
    q = np.random.default_rng(3).standard_normal(q.shape)
    t = 1.3
    qg, _, _ = O.step(po, q, aux, 0.01, t)
    v = -(0.1 * (1.0 + np.cos(np.pi * (t - 1.0) / 1.0)))
    for ibc in (1, 2, 3):
        assert qg[0, 3 - ibc] == q[0, 2 + ibc]
        assert qg[1, 3 - ibc] == 2.0 * v * aux[0, 2 + ibc] - q[1, 2 + ibc]
        assert qg[0, 48 + 2 + ibc] == q[0, 48 + 2] and qg[1, 48 + 2 + ibc] == q[1, 48 + 2]
    # |t - t1| >= tw1: the wall is at rest, a solid wall (bc1.f:130-136)
    qs, dqs, cs = O.step(po, q, aux, 0.01, 2.5)
    pw = cases.stegoton_wall(mx=48, mthbc=(3, 1))[0]
    pw.bc_user = 0
    qw, dqw, cw = O.step(pw, q, aux, 0.01, 2.5)
    assert np.array_equal(qs, qw) and np.array_equal(dqs, dqw) and cs == cw


def test_user_bc_switch_to_periodic():
    """bc1.f:31-45: a stage time in (5 tw1, 5 tw1 + 1) makes both sides
    periodic, q and aux ghosts alike; outside the window nothing changes."""
    po, _, q, aux = cases.stegoton_wall(mx=48)
    rng = np.random.default_rng(4)
    q = rng.standard_normal(q.shape)
    aux = aux.copy()
    aux[:, :3] = rng.uniform(1.0, 4.0, (3, 3))   # ghost aux that differs from the periodic image
    aux[:, -3:] = rng.uniform(1.0, 4.0, (3, 3))
    aux[2] = 0.0
    qg, dq, _ = O.step(po, q, aux, 0.01, 5.5)
    pp = cases.stegoton_wall(mx=48, mthbc=(2, 2))[0]
    pp.bc_user = 0
    auxp = aux.copy()
    auxp[:, :3], auxp[:, -3:] = aux[:, -6:-3], aux[:, 3:6]
    qp, dqp, _ = O.step(pp, q, auxp, 0.01, 5.5)
    assert np.array_equal(qg, qp) and np.array_equal(dq, dqp)
    # a run across the window ends switched; one that stops before does not
    run = dict(tstart=0.0, dt_initial=0.02, cfl_max=2.5, cfl_desired=2.45, time_integrator=4)
    _, r1 = O.sharpclaw(po, np.zeros_like(q), cases.stegoton_wall(mx=48)[3], tend=4.0, **run)
    _, r2 = O.sharpclaw(po, np.zeros_like(q), cases.stegoton_wall(mx=48)[3], tend=5.6, **run)
    assert r1.bc_switched == 0 and r2.bc_switched == 1


def test_oscillating_wall_launches_a_pulse():
    """From rest, the wall motion of 0 < t < 2 puts a pulse into the medium;
    vwall = -a1 g0 < 0 pulls the wall away (bc1.f:59, "negative for
    expansion"), so the strain is mostly positive; by t = 3 the front has travelled
    about 3 (c = 1 in both layers) and the right part is still at rest."""
    po, _, q, aux = cases.stegoton_wall(mx=288)
    qf, res = O.sharpclaw(po, q, aux, tstart=0.0, tend=3.0, dt_initial=0.01, cfl_max=2.5,
                          cfl_desired=2.45, time_integrator=4)
    assert res.info == 0 and res.rejected == 0 and res.bc_switched == 0
    x = (np.arange(288) + 0.5) * po.dx
    eps = qf[0, 3:-3]
    assert eps.max() > 0.005 and eps.max() > 10 * -eps.min()
    assert np.abs(eps[x > 4.5]).max() < 1e-5 * eps.max()


def test_time_reversal_returns_the_pulse():
    """apps/elasticity/stegoton/b4step1.f negates the momentum once, at the
    first step with t + 1e-10 >= trtime.  In a homogeneous medium at strain
    1e-4 (linear), periodic, with dt = 1/32 so a step starts exactly at
    trtime = 5, the wave runs back and at t = 10 the initial pulse is
    restored to 5e-7 (without the flip it has moved away: error 1)."""
    po, _, q, _ = cases.stegoton(mx=600, amp=1e-4, mthbc=(2, 2))
    aux = np.ascontiguousarray(np.stack([np.ones(606), np.ones(606), np.zeros(606)]))
    run = dict(tstart=0.0, tend=10.0, dt_initial=1 / 32, cfl_max=2.5, cfl_desired=2.45, dt_variable=0,
               time_integrator=4)
    po.b4step, po.trtime = 2, 5.0
    qf, r = O.sharpclaw(po, q, aux, **run)
    scale = np.abs(q[0, 3:-3]).max()
    assert r.info == 0
    assert np.abs(qf[0, 3:-3] - q[0, 3:-3]).max() <= 2e-6 * scale
    assert np.abs(qf[1, 3:-3]).max() <= 2e-7 * scale
    po.b4step = 0
    qn, _ = O.sharpclaw(po, q, aux, **run)
    assert np.abs(qn[0, 3:-3] - q[0, 3:-3]).max() >= 0.5 * scale


def _weno5_written(q):
    """src/reconstruct.f90:77-143 written out in Python floats (IEEE double,
    no fused multiply-add), in the source's evaluation order: the REAL(4)
    literals 13., 3., 6., 0.5, 0.25, 12. are exact, `x**2` is x*x,
    epweno = 1.e-36 is the REAL(4) value widened (reconstruct.f90:6).
    Fortran index i (1-based) is Python index i-1."""
    eps = float(np.float32(1e-36))
    mx2 = len(q)
    qf = lambda i: float(q[i - 1])
    d = {i: qf(i) - qf(i - 1) for i in range(2, mx2 + 1)}
    d[1] = float("nan")   # dq1m(1) is never assigned in the reference: qr(2) (a ghost interface) is undefined
    ql = [0.0] * mx2
    qr = [0.0] * mx2
    mbc = 3
    for m1 in (1, 2):
        im = 1 if m1 == 1 else -1
        ione, inone, intwo = im, -im, -2 * im
        for i in range(mbc, mx2 - mbc + 2):
            t1 = im * (d[i + intwo] - d[i + inone])
            t2 = im * (d[i + inone] - d[i])
            t3 = im * (d[i] - d[i + ione])
            x1 = d[i + intwo] - 3.0 * d[i + inone]
            x2 = d[i + inone] + d[i]
            x3 = 3.0 * d[i] - d[i + ione]
            tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1)
            tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2)
            tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3)
            tt1 = (eps + tt1) * (eps + tt1)
            tt2 = (eps + tt2) * (eps + tt2)
            tt3 = (eps + tt3) * (eps + tt3)
            s1 = tt2 * tt3
            s2 = (6.0 * tt1) * tt3
            s3 = (3.0 * tt1) * tt2
            t0 = 1.0 / ((s1 + s2) + s3)
            s1 = s1 * t0
            s3 = s3 * t0
            uu = (s1 * (t2 - t1) + (0.5 * s3 - 0.25) * (t3 - t2)) / 3.0 \
                + ((-qf(i - 2) + 7.0 * (qf(i - 1) + qf(i))) - qf(i + 1)) / 12.0
            if m1 == 1:
                qr[i - 2] = uu      # qr(i-1) = uu(i,1)
            else:
                ql[i - 1] = uu      # ql(i) = uu(i,2)
    return ql, qr


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_weno5_matches_the_written_formulas_bit_for_bit(seed):
    """The oracle's componentwise WENO5 against the reference formulas
    written out independently above, on a smooth line, a jump and noise:
    every reconstructed value identical to the last bit."""
    rng = np.random.default_rng(seed)
    mx2 = 16
    x = np.linspace(0.0, 1.0, mx2)
    lines = [np.sin(2 * np.pi * x) + 0.1 * x, np.where(x < 0.5, 1.0, 0.125), rng.standard_normal(mx2)]
    q = np.stack(lines)
    ql, qr = O.weno5(q)
    for m in range(q.shape[0]):
        wl, wr = _weno5_written(q[m])
        for i in range(3, mx2 - 1):          # ql(i), i = mbc .. mx2-mbc+1 (1-based)
            assert ql[m, i - 1] == wl[i - 1], (m, i)
        for i in range(3, mx2 - 2):          # qr(i), i = mbc .. mx2-mbc (qr(2) is undefined, see above)
            assert qr[m, i - 1] == wr[i - 1], (m, i)


def test_euler_roe_waves_matches_the_written_formulas_bit_for_bit():
    """The oracle's Euler Riemann solver (Roe averages, wave strengths,
    waves and speeds) against apps/euler/shockentropy/rp1eu.f:44-86 written
    out independently in Python floats, in the source's evaluation order
    (`x**2` as x*x, products and quotients left to right, dsqrt correctly
    rounded): identical to the last bit at every interface."""
    import math
    rng = np.random.default_rng(21)
    n = 24
    p = O.make_params(mx=n - 6, meqn=3, mwaves=3, dx=0.1, rp=O.RP_EULER, mthbc=(1, 1))
    gamma1 = p.gamma - 1.0
    rho = rng.uniform(0.2, 3.0, n)
    u = rng.uniform(-2.0, 2.0, n)
    pr = rng.uniform(0.2, 3.0, n)
    q = np.stack([rho, rho * u, pr / 0.4 + 0.5 * rho * u * u])
    ql = q.copy()
    qr = np.roll(q, 1, axis=1) * 1.01          # a jump at every interface
    wave, s, _, _ = O.rp(p, ql, qr)
    for i in range(1, n):
        l1, l2, l3 = (float(v) for v in qr[:, i - 1])
        r1, r2, r3 = (float(v) for v in ql[:, i])
        rhsqrtl, rhsqrtr = math.sqrt(l1), math.sqrt(r1)
        pl = gamma1 * (l3 - (0.5 * (l2 * l2)) / l1)
        prr = gamma1 * (r3 - (0.5 * (r2 * r2)) / r1)
        rhsq2 = rhsqrtl + rhsqrtr
        ui = (l2 / rhsqrtl + r2 / rhsqrtr) / rhsq2
        enth = ((l3 + pl) / rhsqrtl + (r3 + prr) / rhsqrtr) / rhsq2
        ai = math.sqrt(gamma1 * (enth - 0.5 * (ui * ui)))
        d1, d2, d3 = r1 - l1, r2 - l2, r3 - l3
        a2 = (gamma1 / (ai * ai)) * (((enth - ui * ui) * d1 + ui * d2) - d3)
        a3 = ((d2 + (ai - ui) * d1) - ai * a2) / (2.0 * ai)
        a1 = (d1 - a2) - a3
        want_w = [[a1, a1 * (ui - ai), a1 * (enth - ui * ai)],
                  [a2, a2 * ui, (a2 * 0.5) * (ui * ui)],
                  [a3, a3 * (ui + ai), a3 * (enth + ui * ai)]]
        want_s = [ui - ai, ui, ui + ai]
        for mw in range(3):
            assert s[mw, i] == want_s[mw], (i, mw)
            for m in range(3):
                assert wave[mw, m, i] == want_w[mw][m], (i, mw, m)


def test_weno5_char_matches_the_written_formulas_bit_for_bit():
    """The oracle's characteristic-wise WENO5 against src/reconstruct.f90:
    146-241 written out independently (projection sums from 0 in component
    order, the same WENO algebra on the projections, back-projection added
    field by field), with arbitrary per-interface eigenvector matrices:
    identical to the last bit at every interface the reference defines
    (interface 3 reads projections hh(3,:) that the reference never sets)."""
    import ctypes
    rng = np.random.default_rng(5)
    meqn, mx2 = 3, 18
    q = rng.standard_normal((meqn, mx2)) + np.linspace(0, 2, mx2)
    evl = rng.standard_normal((meqn, meqn, mx2))     # evl(i, ip, m) at [m, ip, i]
    evr = rng.standard_normal((meqn, meqn, mx2))     # evr(i, m, ip) at [ip, m, i]
    ql = np.zeros((meqn, mx2))
    qr = np.zeros((meqn, mx2))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert O.lib().ocl_weno5_char(mx2, meqn, dp(q), dp(evl), dp(evr), dp(ql), dp(qr)) == 0
    eps = float(np.float32(1e-36))
    Q = lambda i, m: float(q[m - 1, i - 1])
    EL = lambda i, ip, m: float(evl[m - 1, ip - 1, i - 1])
    ER = lambda i, m, ip: float(evr[ip - 1, m - 1, i - 1])
    dq = {(i, m): Q(i, m) - Q(i - 1, m) for m in range(1, meqn + 1) for i in range(2, mx2 + 1)}
    wl, wr = {}, {}
    for m in range(1, meqn + 1):
        for i in range(3, mx2):
            c = ((-Q(i - 2, m)) + 7.0 * (Q(i - 1, m) + Q(i, m))) - Q(i + 1, m)
            wr[(i - 1, m)] = c / 12.0
            wl[(i, m)] = wr[(i - 1, m)]
    for ip in range(1, meqn + 1):
        hh = {}
        for m2 in range(-2, 3):
            for i in range(4, mx2 - 1):
                h = 0.0
                for m in range(1, meqn + 1):
                    h = h + EL(i, ip, m) * dq[(i + m2, m)]
                hh[(i, m2)] = h
        for m2 in range(-2, 3):
            hh[(3, m2)] = float("nan")
        uu = {}
        for m1 in (1, 2):
            im = 1 if m1 == 1 else -1
            ione, inone, intwo = im, -im, -2 * im
            for i in range(3, mx2 - 1):
                t1 = im * (hh[(i, intwo)] - hh[(i, inone)])
                t2 = im * (hh[(i, inone)] - hh[(i, 0)])
                t3 = im * (hh[(i, 0)] - hh[(i, ione)])
                x1 = hh[(i, intwo)] - 3.0 * hh[(i, inone)]
                x2 = hh[(i, inone)] + hh[(i, 0)]
                x3 = 3.0 * hh[(i, 0)] - hh[(i, ione)]
                tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1)
                tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2)
                tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3)
                tt1 = (eps + tt1) * (eps + tt1)
                tt2 = (eps + tt2) * (eps + tt2)
                tt3 = (eps + tt3) * (eps + tt3)
                s1 = tt2 * tt3
                s2 = (6.0 * tt1) * tt3
                s3 = (3.0 * tt1) * tt2
                t0 = 1.0 / ((s1 + s2) + s3)
                s1 = s1 * t0
                s3 = s3 * t0
                uu[(i, m1)] = (s1 * (t2 - t1) + (0.5 * s3 - 0.25) * (t3 - t2)) / 3.0
        for m in range(1, meqn + 1):
            for i in range(3, mx2 - 1):
                wr[(i - 1, m)] = wr[(i - 1, m)] + ER(i, m, ip) * uu[(i, 1)]
                wl[(i, m)] = wl[(i, m)] + ER(i, m, ip) * uu[(i, 2)]
    for m in range(1, meqn + 1):
        for i in range(4, mx2 - 1):          # interfaces 4 .. mx2-2: qr(i-1), ql(i)
            assert qr[m - 1, i - 2] == wr[(i - 1, m)], (m, i)
            assert ql[m - 1, i - 1] == wl[(i, m)], (m, i)


def _euler_roe_written(l, r, gamma):
    """rp1eu.f:44-86 at one interface (left state l = qr(i-1), right r =
    ql(i)): the waves [mw][m] and speeds, in the source's order."""
    import math
    gamma1 = gamma - 1.0
    l1, l2, l3 = l
    r1, r2, r3 = r
    rhsqrtl, rhsqrtr = math.sqrt(l1), math.sqrt(r1)
    pl = gamma1 * (l3 - (0.5 * (l2 * l2)) / l1)
    prr = gamma1 * (r3 - (0.5 * (r2 * r2)) / r1)
    rhsq2 = rhsqrtl + rhsqrtr
    u = (l2 / rhsqrtl + r2 / rhsqrtr) / rhsq2
    enth = ((l3 + pl) / rhsqrtl + (r3 + prr) / rhsqrtr) / rhsq2
    a = math.sqrt(gamma1 * (enth - 0.5 * (u * u)))
    d1, d2, d3 = r1 - l1, r2 - l2, r3 - l3
    a2 = (gamma1 / (a * a)) * (((enth - u * u) * d1 + u * d2) - d3)
    a3 = ((d2 + (a - u) * d1) - a * a2) / (2.0 * a)
    a1 = (d1 - a2) - a3
    w = [[a1, a1 * (u - a), a1 * (enth - u * a)],
         [a2, a2 * u, (a2 * 0.5) * (u * u)],
         [a3, a3 * (u + a), a3 * (enth + u * a)]]
    return w, [u - a, u, u + a]


def _euler_efix_written(l, r, w, s, gamma):
    """rp1eu.f:116-213 (Harten-Hyman entropy fix) at one interface: amdq,
    apdq and the branch taken for the 1- and 3-waves."""
    import math
    gamma1 = gamma - 1.0

    def sound(rho, mom, en):
        p = gamma1 * (en - (0.5 * (mom * mom)) / rho)
        x = (gamma * p) / rho
        return math.sqrt(x) if x >= 0.0 else float("nan")   # dsqrt of a negative: NaN

    amdq = [0.0, 0.0, 0.0]
    branch = "supersonic"
    cim1 = sound(*l)
    s0 = l[1] / l[0] - cim1
    if not (s0 >= 0.0 and s[0] > 0.0):
        rho1, rhou1, en1 = l[0] + w[0][0], l[1] + w[0][1], l[2] + w[0][2]
        s1 = rhou1 / rho1 - sound(rho1, rhou1, en1)
        if s0 < 0.0 and s1 > 0.0:
            sfract, branch = (s0 * (s1 - s[0])) / (s1 - s0), "transonic-1"
        elif s[0] < 0.0:
            sfract, branch = s[0], "left-1"
        else:
            sfract, branch = 0.0, "right-1"
        amdq = [sfract * w[0][m] for m in range(3)]
        if not (s[1] >= 0.0):
            amdq = [amdq[m] + s[1] * w[1][m] for m in range(3)]
            ci = sound(*r)
            s3 = r[1] / r[0] + ci
            rho2, rhou2, en2 = r[0] - w[2][0], r[1] - w[2][1], r[2] - w[2][2]
            s2 = rhou2 / rho2 + sound(rho2, rhou2, en2)
            sf3 = None
            if s2 < 0.0 and s3 > 0.0:
                sf3, branch = (s2 * (s3 - s[2])) / (s3 - s2), branch + ",transonic-3"
            elif s[2] < 0.0:
                sf3, branch = s[2], branch + ",left-3"
            if sf3 is not None:
                amdq = [amdq[m] + sf3 * w[2][m] for m in range(3)]
    apdq = []
    for m in range(3):
        df = 0.0
        for mw in range(3):
            df = df + s[mw] * w[mw][m]
        apdq.append(df - amdq[m])
    return amdq, apdq, branch


def test_euler_entropy_fix_matches_the_written_formulas_bit_for_bit():
    """The oracle's Euler solver with the Harten-Hyman entropy fix (the C2
    headline's solver) against rp1eu.f:44-213 written out above: amdq and
    apdq identical to the last bit at every interface of lines built to hit
    the transonic 1- and 3-rarefactions as well as sub- and supersonic
    interfaces."""
    rng = np.random.default_rng(17)
    n = 400
    p = O.make_params(mx=n - 6, meqn=3, mwaves=3, dx=0.1, rp=O.RP_EULER, mthbc=(1, 1), efix=1)
    rho = rng.uniform(0.3, 2.0, n)
    pr = rng.uniform(0.3, 2.0, n)
    c = np.sqrt(1.4 * pr / rho)
    u = c * rng.uniform(-1.6, 1.6, n)            # Mach numbers across the sonic points
    q = np.stack([rho, rho * u, pr / 0.4 + 0.5 * rho * u * u])
    ql = q.copy()
    qr = 0.75 * np.roll(q, 1, axis=1) + 0.25 * q   # moderate jumps: physical intermediate states
    _, _, am, ap = O.rp(p, ql, qr)
    branches = set()
    for i in range(1, n):
        left = tuple(float(v) for v in qr[:, i - 1])
        right = tuple(float(v) for v in ql[:, i])
        w, s = _euler_roe_written(left, right, p.gamma)
        wam, wap, br = _euler_efix_written(left, right, w, s, p.gamma)
        branches.add(br)
        for m in range(3):
            assert am[m, i] == wam[m], (i, m, br)
            assert ap[m, i] == wap[m], (i, m, br)
    assert any("transonic-1" in b for b in branches) and any("transonic-3" in b for b in branches)
    assert "supersonic" in branches


def test_ssp104_step_matches_the_written_integrator_bit_for_bit():
    """The oracle's SSPRK(10,4) step (the C2 headline integrator) against
    ts_ssp104 (src/sharpclaw.f90:380-464) written out with whole-array
    numpy operations in the source's order around the oracle's own step()
    (bc + flux1 -> dt*L(q)): identical to the last bit on a Shu-Osher line
    with the entropy-fixed Roe solver and char-wise WENO5."""
    po, _, q, aux = cases.shu_osher(mx=200)
    po.char_decomp = 2
    dt = 0.002
    sixth = 1.0 / 6.0
    qold = O.bc(po, q)
    qq = qold.copy()
    for _ in range(4):                                   # stages 1-4: q = q + 1/6 r1
        qq, r1, _ = O.step(po, qq, aux, dt)
        qq = qq + sixth * r1
    qq, r1, _ = O.step(po, qq, aux, dt)                  # stage 5
    r2 = qq + sixth * r1
    r1 = 0.04 * qold + 0.36 * r2
    qq = 0.6 * qold + 0.4 * r2
    for _ in range(4):                                   # stages 6-9: q = q + 1/6 r2
        qq, r2, _ = O.step(po, qq, aux, dt)
        qq = qq + sixth * r2
    qq, r2, _ = O.step(po, qq, aux, dt)                  # stage 10
    qq = (r1 + 0.6 * qq) + 0.1 * r2
    got, _ = O.rk_step(po, 4, qold, aux, dt)
    assert np.array_equal(got[:, 3:-3], qq[:, 3:-3])


def test_flux1_matches_the_written_assembly_bit_for_bit():
    """The oracle's flux1 for the C2 configuration (char-wise WENO5,
    tfluct_solver = 0: the second Riemann solve inside each cell after the
    in-place swap of src/flux1.f90:163-168) against src/flux1.f90:55-187
    written out here around the oracle's own evec, weno5_char and rp: dq and
    the CFL number identical to the last bit."""
    import ctypes
    po, _, q, aux = cases.shu_osher(mx=120)
    po.char_decomp = 2
    po.tfluct_solver = 0
    dt = 0.003
    qb = O.bc(po, q)
    _, dq_oracle, cfl_oracle = O.step(po, qb, aux, dt)
    meqn, mx2 = qb.shape
    mx = mx2 - 6
    dtdx = dt / po.dx
    evl, evr = O.evec(po, qb)
    ql = np.zeros_like(qb)
    qr = np.zeros_like(qb)
    dp = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert O.lib().ocl_weno5_char(mx2, meqn, dp(qb), dp(evl), dp(evr), dp(ql), dp(qr)) == 0
    _, s, amdq, apdq = O.rp(po, ql, qr)
    cfl = 0.0
    for mw in range(s.shape[0]):
        for i in range(1, mx + 2):                    # interfaces 1 .. mx+1 (array index i+2)
            k = i + 2
            cfl = max(cfl, dtdx * float(s[mw, k]), -dtdx * float(s[mw, k]))
    ql2, qr2 = ql.copy(), qr.copy()
    for k in range(1, mx2):                           # i = 1-mbc+1 .. mx+mbc, in order
        qr2[:, k - 1] = ql2[:, k]
        ql2[:, k] = qr2[:, k]
    _, _, amdq2, apdq2 = O.rp(po, ql2, qr2)
    dq = np.zeros_like(qb)
    for k in range(3, mx + 3):                        # cells 1 .. mx
        dq[:, k] = dq[:, k] - dtdx * (((amdq[:, k + 1] + apdq[:, k]) + amdq2[:, k]) + apdq2[:, k])
    assert cfl == cfl_oracle
    assert np.array_equal(dq[:, 3:-3], dq_oracle[:, 3:-3])


def test_flux2_matches_the_written_sweeps_bit_for_bit():
    """The oracle's 2-D step (C3's shallow-water configuration: char-wise
    WENO5, Roe rpn2 + tfluct) against src/2d/flux2.f90:28-92 written out
    here around the oracle's own 1-D flux1: x sweeps over the rows
    j = 0..ny+1, then y sweeps over the columns i = 0..nx+1 (the ghost lines
    count in the CFL number), dq accumulated row sweep first: dq and the
    CFL number identical to the last bit."""
    import ctypes
    po, _, q, aux = cases.radial_dam(n=20)
    dt = 0.004
    qb = O.bc(po, q)
    _, dq_oracle, cfl_oracle = O.step(po, qb, aux, dt)
    meqn, my2, mx2 = qb.shape
    nx, ny = mx2 - 6, my2 - 6
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    dq = np.zeros_like(qb)
    cfl = 0.0
    for jj in range(2, ny + 4):                       # rows j = 0 .. ny+1
        q1d = np.ascontiguousarray(qb[:, jj, :])
        dq1d = np.zeros_like(q1d)
        c1 = ctypes.c_double(0.0)
        assert O.lib().ocl_flux1(ctypes.byref(po), dp(q1d), dp(dq1d), None, dt, ctypes.byref(c1), 1, nx) == 0
        cfl = max(cfl, c1.value)
        dq[:, jj, 3:nx + 3] = dq[:, jj, 3:nx + 3] + dq1d[:, 3:nx + 3]
    for ii in range(2, nx + 4):                       # columns i = 0 .. nx+1
        q1d = np.ascontiguousarray(qb[:, :, ii])
        dq1d = np.zeros_like(q1d)
        c1 = ctypes.c_double(0.0)
        assert O.lib().ocl_flux1(ctypes.byref(po), dp(q1d), dp(dq1d), None, dt, ctypes.byref(c1), 2, ny) == 0
        cfl = max(cfl, c1.value)
        dq[:, 3:ny + 3, ii] = dq[:, 3:ny + 3, ii] + dq1d[:, 3:ny + 3]
    assert cfl == cfl_oracle
    assert np.array_equal(dq[:, 3:-3, 3:-3], dq_oracle[:, 3:-3, 3:-3])


@pytest.mark.parametrize("ixy", [1, 2])
def test_sw2d_roe_matches_the_written_formulas_bit_for_bit(ixy):
    """The oracle's 2-D shallow-water Riemann solver (C3) against
    apps/shallowWater/2dRadialDam/rpn2sw.f:60-143 written out here (normal
    and tangential momentum chosen by ixy, no entropy fix as in the app):
    waves, speeds, amdq and apdq identical to the last bit."""
    import math
    rng = np.random.default_rng(31 + ixy)
    n = 40
    p = O.make_params(ndim=2, mx=n - 6, my=n - 6, meqn=3, mwaves=3, dx=0.1, dy=0.1, rp=O.RP_SW2D,
                      grav=1.0, mthbc=(1, 1, 1, 1))
    h = rng.uniform(0.5, 2.0, n)
    q = np.stack([h, h * rng.uniform(-1.5, 1.5, n), h * rng.uniform(-1.5, 1.5, n)])
    ql = q.copy()
    qr = 0.7 * np.roll(q, 1, axis=1) + 0.3 * q
    wave, s, am, ap = O.rp(p, ql, qr, ixy=ixy)
    mu, mv = (1, 2) if ixy == 1 else (2, 1)          # 0-based momentum components
    g = p.grav
    for i in range(1, n):
        l = [float(v) for v in qr[:, i - 1]]
        r = [float(v) for v in ql[:, i]]
        hh = (l[0] + r[0]) * 0.5
        hsqrtl, hsqrtr = math.sqrt(l[0]), math.sqrt(r[0])
        hsq2 = hsqrtl + hsqrtr
        u = (l[mu] / hsqrtl + r[mu] / hsqrtr) / hsq2
        v = (l[mv] / hsqrtl + r[mv] / hsqrtr) / hsq2
        a = math.sqrt(g * hh)
        d1, d2, d3 = r[0] - l[0], r[mu] - l[mu], r[mv] - l[mv]
        a1 = ((u + a) * d1 - d2) * (0.5 / a)
        a2 = -v * d1 + d3
        a3 = (-(u - a) * d1 + d2) * (0.5 / a)
        w = [[0.0] * 3 for _ in range(3)]
        w[0][0], w[0][mu], w[0][mv] = a1, a1 * (u - a), a1 * v
        w[1][0], w[1][mu], w[1][mv] = 0.0, 0.0, a2
        w[2][0], w[2][mu], w[2][mv] = a3, a3 * (u + a), a3 * v
        sp = [u - a, u, u + a]
        for m in range(3):
            amdq, apdq = 0.0, 0.0
            for mw in range(3):
                if sp[mw] < 0.0:
                    amdq = amdq + sp[mw] * w[mw][m]
                else:
                    apdq = apdq + sp[mw] * w[mw][m]
            assert am[m, i] == amdq and ap[m, i] == apdq, (i, m)
            for mw in range(3):
                assert wave[mw, m, i] == w[mw][m], (i, mw, m)
        for mw in range(3):
            assert s[mw, i] == sp[mw], (i, mw)


def test_ssp33_step_matches_the_written_integrator_bit_for_bit():
    """The oracle's SSPRK(3,3) step (C1, C3, C4, C5) against ts_ssp33
    (src/sharpclaw.f90:337-376) written out around the oracle's step()."""
    po, _, q, aux = cases.advection(mx=150)
    dt = 0.004
    qold = O.bc(po, q)
    qq, r1, _ = O.step(po, qold, aux, dt)
    qq = qq + r1
    qq, r1, _ = O.step(po, qq, aux, dt, t=dt)
    qq = 0.75 * qold + 0.25 * (qq + r1)
    qq, r1, _ = O.step(po, qq, aux, dt, t=0.5 * dt)
    qq = (qold + 2.0 * (qq + r1)) / 3.0
    got, _ = O.rk_step(po, 3, qold, aux, dt)
    assert np.array_equal(got[:, 3:-3], qq[:, 3:-3])


@pytest.mark.parametrize("ixy", [1, 2])
def test_sw2d_tfluct_matches_the_written_formulas_bit_for_bit(ixy):
    """The oracle's shallow-water total fluctuation inside each cell (C3's
    tfluct_solver = 1) against apps/shallowWater/2dRadialDam/tfluct1sw.f:
    78-140 written out here: the Roe solve from ql(i) to qr(i) of the same
    cell, adq = amdq + apdq, identical to the last bit."""
    import ctypes
    import math
    rng = np.random.default_rng(41 + ixy)
    n = 30
    p = O.make_params(ndim=2, mx=n - 6, my=n - 6, meqn=3, mwaves=3, dx=0.1, dy=0.1, rp=O.RP_SW2D,
                      grav=1.0, mthbc=(1, 1, 1, 1))
    hl = rng.uniform(0.5, 2.0, n)
    ql = np.stack([hl, hl * rng.uniform(-1.5, 1.5, n), hl * rng.uniform(-1.5, 1.5, n)])
    qr = ql * rng.uniform(0.8, 1.25, (3, n))
    s = np.zeros((3, n))
    adq = np.zeros((3, n))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert O.lib().ocl_tfluct(ctypes.byref(p), ixy, n - 6, dp(ql), dp(qr), None, None, dp(s), dp(adq)) == 0
    mu, mv = (1, 2) if ixy == 1 else (2, 1)
    g = p.grav
    for i in range(1, n):
        l = [float(v) for v in ql[:, i]]
        r = [float(v) for v in qr[:, i]]
        hh = (l[0] + r[0]) * 0.5
        hsqrtl, hsqrtr = math.sqrt(l[0]), math.sqrt(r[0])
        hsq2 = hsqrtl + hsqrtr
        u = (l[mu] / hsqrtl + r[mu] / hsqrtr) / hsq2
        v = (l[mv] / hsqrtl + r[mv] / hsqrtr) / hsq2
        a = math.sqrt(g * hh)
        d1, d2, d3 = r[0] - l[0], r[mu] - l[mu], r[mv] - l[mv]
        a1 = ((u + a) * d1 - d2) * (0.5 / a)
        a2 = -v * d1 + d3
        a3 = (-(u - a) * d1 + d2) * (0.5 / a)
        w = [[0.0] * 3 for _ in range(3)]
        w[0][0], w[0][mu], w[0][mv] = a1, a1 * (u - a), a1 * v
        w[1][0], w[1][mu], w[1][mv] = 0.0, 0.0, a2
        w[2][0], w[2][mu], w[2][mv] = a3, a3 * (u + a), a3 * v
        sp = [u - a, u, u + a]
        for m in range(3):
            amdq, apdq = 0.0, 0.0
            for mw in range(3):
                if sp[mw] < 0.0:
                    amdq = amdq + sp[mw] * w[mw][m]
                else:
                    apdq = apdq + sp[mw] * w[mw][m]
            assert adq[m, i] == amdq + apdq, (i, m)


def test_acoustics_interface_solvers_matches_the_written_formulas_bit_for_bit():
    """The oracle's variable-coefficient acoustics Riemann solver and total
    fluctuation (the reference's known-answer app) against
    apps/acoustics/1d/interface/rp1acv.f:42-81 and tfluct1acv.f:42-81
    written out here (impedance aux(:,1), sound speed aux(:,2); the total
    fluctuation uses the cell's own coefficients on both sides): waves,
    speeds, amdq, apdq and adq identical to the last bit."""
    import ctypes
    rng = np.random.default_rng(51)
    n = 30
    p = O.make_params(meqn=2, mwaves=2, maux=2, mx=n - 6, dx=0.1, rp=O.RP_ACOUSTICS1D, mthbc=(1, 1))
    aux = np.stack([rng.uniform(0.5, 3.0, n), rng.uniform(0.5, 2.0, n)])
    ql = rng.standard_normal((2, n))
    qr = rng.standard_normal((2, n))
    wave, s, am, ap = O.rp(p, ql, qr, aux, aux)
    sf = np.zeros((2, n))
    adq = np.zeros((2, n))
    dp = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert O.lib().ocl_tfluct(ctypes.byref(p), 1, n - 6, dp(ql), dp(qr), dp(aux), dp(aux), dp(sf), dp(adq)) == 0
    for i in range(1, n):
        # rp1acv: interface i, left qr(i-1) with auxr(i-1), right ql(i) with auxl(i)
        d1, d2 = float(ql[0, i]) - float(qr[0, i - 1]), float(ql[1, i]) - float(qr[1, i - 1])
        zi, zim = float(aux[0, i]), float(aux[0, i - 1])
        a1 = (-d1 + zi * d2) / (zim + zi)
        a2 = (d1 + zim * d2) / (zim + zi)
        w = [[-a1 * zim, a1], [a2 * zi, a2]]
        sp = [-float(aux[1, i - 1]), float(aux[1, i])]
        for m in range(2):
            assert wave[0, m, i] == w[0][m] and wave[1, m, i] == w[1][m], (i, m)
            assert am[m, i] == sp[0] * w[0][m] and ap[m, i] == sp[1] * w[1][m], (i, m)
        assert s[0, i] == sp[0] and s[1, i] == sp[1], i
        # tfluct1acv: inside cell i, from ql(i) to qr(i), both sides with aux(i)
        d1, d2 = float(qr[0, i]) - float(ql[0, i]), float(qr[1, i]) - float(ql[1, i])
        zi = zim = float(aux[0, i])
        a1 = (-d1 + zi * d2) / (zim + zi)
        a2 = (d1 + zim * d2) / (zim + zi)
        w = [[-a1 * zim, a1], [a2 * zi, a2]]
        sp = [-float(aux[1, i]), float(aux[1, i])]
        for m in range(2):
            assert adq[m, i] == sp[0] * w[0][m] + sp[1] * w[1][m], (i, m)


@pytest.mark.parametrize("mthbc", [(1, 1), (2, 2), (3, 3), (1, 3), (3, 1)])
def test_bc1_matches_the_written_formulas(mthbc):
    """The oracle's 1-D ghost fill against src/1d/bc1.f90:40-109 written out
    here: extrapolation copies the end cell, periodic wraps, a wall mirrors
    with the second component negated; interior untouched."""
    rng = np.random.default_rng(61)
    mx, mbc = 9, 3
    p = O.make_params(meqn=2, mwaves=2, mx=mx, dx=0.1, rp=O.RP_ACOUSTICS_CONST, rho=1.0, bulk=1.0,
                      mthbc=mthbc)
    q = rng.standard_normal((2, mx + 2 * mbc))
    got = O.bc(p, q)
    want = q.copy()
    Q = lambda i: i + mbc - 1                 # Fortran cell index -> array index
    for m in range(2):
        for ibc in range(1, mbc + 1):
            if mthbc[0] == 1:
                want[m, Q(1 - ibc)] = want[m, Q(1)]
            elif mthbc[0] == 2:
                want[m, Q(1 - ibc)] = want[m, Q(mx + 1 - ibc)]
            else:
                want[m, Q(1 - ibc)] = want[m, Q(ibc)]
    if mthbc[0] == 3:
        for ibc in range(1, mbc + 1):
            want[1, Q(1 - ibc)] = -want[1, Q(ibc)]
    for m in range(2):
        for ibc in range(1, mbc + 1):
            if mthbc[1] == 1:
                want[m, Q(mx + ibc)] = want[m, Q(mx)]
            elif mthbc[1] == 2:
                want[m, Q(mx + ibc)] = want[m, Q(ibc)]
            else:
                want[m, Q(mx + ibc)] = want[m, Q(mx + 1 - ibc)]
    if mthbc[1] == 3:
        for ibc in range(1, mbc + 1):
            want[1, Q(mx + ibc)] = -want[1, Q(mx + 1 - ibc)]
    assert np.array_equal(got, want)


def _fill_side(a, axis, side, kind, n, mbc, neg_comp):
    """One side of bc1/bc2 along `axis` of a (meqn, ..., n+2mbc) slab: the
    written rules of src/2d/bc2.f90 (extrapolation, periodic, wall with
    component neg_comp negated), over every line of the other axis."""
    def sl(k):
        idx = [slice(None)] * a.ndim
        idx[axis] = k
        return tuple(idx)
    Q = lambda i: i + mbc - 1
    for ibc in range(1, mbc + 1):
        g = Q(1 - ibc) if side == 0 else Q(n + ibc)
        if kind == 1:
            src = Q(1) if side == 0 else Q(n)
        elif kind == 2:
            src = Q(n + 1 - ibc) if side == 0 else Q(ibc)
        else:
            src = Q(ibc) if side == 0 else Q(n + 1 - ibc)
        a[sl(g)] = a[sl(src)]
        if kind == 3:
            gi = list(sl(g))
            si = list(sl(src))
            gi[0] = si[0] = neg_comp
            a[tuple(gi)] = -a[tuple(si)]


@pytest.mark.parametrize("mthbc", [(1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3), (1, 3, 3, 1), (3, 3, 2, 2)])
def test_bc2_matches_the_written_formulas(mthbc):
    """The oracle's 2-D ghost fill against src/2d/bc2.f90 written out here:
    the x sides first over every row (ghost rows included), then the y sides
    over every column (ghost columns included), so the corners carry the
    y rule applied to the x-filled columns; momentum component 2 negated at
    x walls, 3 at y walls."""
    rng = np.random.default_rng(71)
    nx, ny, mbc = 7, 6, 3
    p = O.make_params(ndim=2, meqn=3, mwaves=3, mx=nx, my=ny, dx=0.1, dy=0.1, rp=O.RP_SW2D,
                      mthbc=mthbc)
    q = rng.standard_normal((3, ny + 2 * mbc, nx + 2 * mbc))
    got = O.bc(p, q)
    want = q.copy()
    _fill_side(want, 2, 0, mthbc[0], nx, mbc, 1)
    _fill_side(want, 2, 1, mthbc[1], nx, mbc, 1)
    _fill_side(want, 1, 0, mthbc[2], ny, mbc, 2)
    _fill_side(want, 1, 1, mthbc[3], ny, mbc, 2)
    assert np.array_equal(got, want)
