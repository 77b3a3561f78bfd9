"""Problem set-ups shared by the oracle and GPU tests (seeded, small)."""
import numpy as np

from oracle import oracle as O
import sharpclaw_b200 as S


def advection(mx=200, seed=1, mthbc=(2, 2), char_decomp=0, tfluct_solver=1):
    """Periodic advection with the C1 initial data: a Gaussian, a square pulse
    and four seeded sinusoids, point values at cell centres."""
    dx = 1.0 / mx
    rng = np.random.default_rng(seed)
    xc = (np.arange(mx) + 0.5) * dx
    q0 = np.exp(-200.0 * (xc - 0.3) ** 2) + ((xc > 0.6) & (xc < 0.8))
    for _ in range(4):
        k = rng.integers(1, 9)
        q0 = q0 + rng.uniform(0, 0.1) * np.sin(2 * np.pi * k * xc)
    q = np.zeros((1, mx + 6))
    q[0, 3:-3] = q0
    kw = dict(mx=mx, dx=dx, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=tfluct_solver)
    po = O.make_params(meqn=1, mwaves=1, rp=O.RP_ADVECTION, u=1.0, **kw)
    ps = S.ClawParams(rp=S.RP_ADVECTION, u=1.0, **kw)
    return po, ps, q, None


def shu_osher(mx=400, gamma=1.4, char_decomp=2, mthbc=(1, 1), perturb=0.0, seed=2):
    """Shu-Osher shock/entropy-wave interaction on [-5, 5]
    (apps/euler/shockentropy/qinit.f:299-323)."""
    xlower, xupper = -5.0, 5.0
    dx = (xupper - xlower) / mx
    xc = xlower + (np.arange(1, mx + 1) - 0.5) * dx
    g1 = gamma - 1.0
    rhol, ul, pl = 3.857143, 2.629369, 10.333333
    rho = np.where(xc < -4.0, rhol, 1.0 + 0.2 * np.sin(5.0 * xc))
    mom = np.where(xc < -4.0, rhol * ul, 0.0)
    en = np.where(xc < -4.0, pl / g1 + 0.5 * rhol * ul ** 2, 1.0 / g1)
    if perturb:
        rng = np.random.default_rng(seed)
        mom = mom + perturb * rng.standard_normal(mx)
    q = np.zeros((3, mx + 6))
    q[0, 3:-3], q[1, 3:-3], q[2, 3:-3] = rho, mom, en
    kw = dict(mx=mx, dx=dx, xlower=xlower, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=0)
    po = O.make_params(meqn=3, mwaves=3, rp=O.RP_EULER, gamma=gamma, **kw)
    ps = S.ClawParams(rp=S.RP_EULER, gamma=gamma, **kw)
    return po, ps, q, None


def riemann(mx=300, rho=(1.0, 0.125), u=(0.0, 0.0), p=(1.0, 0.1), gamma=1.4, char_decomp=0):
    """1-D Euler Riemann problem on [0,1], jump at 0.5, extrapolation bc."""
    dx = 1.0 / mx
    xc = (np.arange(mx) + 0.5) * dx
    left = xc < 0.5
    r = np.where(left, rho[0], rho[1])
    v = np.where(left, u[0], u[1])
    pr = np.where(left, p[0], p[1])
    q = np.zeros((3, mx + 6))
    q[0, 3:-3], q[1, 3:-3], q[2, 3:-3] = r, r * v, pr / (gamma - 1) + 0.5 * r * v * v
    kw = dict(mx=mx, dx=dx, mthbc=(1, 1), char_decomp=char_decomp, tfluct_solver=0)
    po = O.make_params(meqn=3, mwaves=3, rp=O.RP_EULER, gamma=gamma, **kw)
    ps = S.ClawParams(rp=S.RP_EULER, gamma=gamma, **kw)
    return po, ps, q, None


def acoustics1d(mx=200, rho=(1.0, 4.0), c=(1.0, 0.5), char_decomp=0, tfluct_solver=1, mthbc=(2, 2)):
    from acoustics_exact import InterfaceProblem
    ap = InterfaceProblem(rho=rho, c=c)
    dx = 20.0 / mx
    aux = ap.setaux(mx)
    q = ap.qinit(mx, aux)
    kw = dict(mx=mx, dx=dx, xlower=-10.0, mthbc=mthbc, char_decomp=char_decomp,
              tfluct_solver=tfluct_solver)
    po = O.make_params(meqn=2, mwaves=2, maux=2, rp=O.RP_ACOUSTICS1D, **kw)
    ps = S.ClawParams(rp=S.RP_ACOUSTICS1D, **kw)
    return po, ps, q, aux


def stegoton_wall(mx=288, upper=6.0, wall=(1.0, 0.1, 1.0, 0.0, 0.0, 1.0), mthbc=(0, 1), char_decomp=0):
    """apps/elasticity/stegoton as its sharpclaw.data runs it: q = 0, the
    oscillating wall of bc1.f at xlower (mthbc 0) and extrapolation at xupper,
    the switch to periodic when a stage time enters (5 tw1, 5 tw1 + 1).  The
    app's wall (t1 = 10, a1 = 0.1, tw1 = 10 on [0, 150]) is scaled to
    t1 = tw1 = 1 on [0, upper] so the pulse, its travel and the switch fit a
    short run; a1 = 0.1 as the app; 48 cells per layer period as the app's
    mx = 7200.  Layers as setaux.f: ix = xcell truncates toward zero, so the
    ghost cells left of x = 0 are layer A, the mirror image of cells 1..3 --
    a wall between unlike materials (floor instead of truncation) feeds
    energy into the reflected wave and the run blows up."""
    po, ps, q, aux = stegoton(mx=mx, char_decomp=char_decomp, mthbc=mthbc, amp=0.0)
    dx = upper / mx
    xa = (np.arange(-3, mx + 3) + 0.5) * dx
    frac = xa - np.trunc(xa)
    rho = np.where(frac < 0.5, 1.0, 4.0)
    aux = np.ascontiguousarray(np.stack([rho, rho.copy(), np.zeros_like(xa)]))
    po = O.make_params(meqn=2, mwaves=2, maux=3, rp=O.RP_STEGOTON, mx=mx, dx=dx, xlower=0.0, mthbc=mthbc,
                       char_decomp=char_decomp, tfluct_solver=1, bc_user=1, wall=wall)
    ps = S.ClawParams(rp=S.RP_STEGOTON, mx=mx, dx=dx, xlower=0.0, mthbc=mthbc, char_decomp=char_decomp,
                      tfluct_solver=1, bc_user=S.BC_USER_OSCILLATING_WALL, wall=wall)
    return po, ps, np.zeros((2, mx + 6)), aux


def radial_dam(n=48, noise=1e-3, seed=3, char_decomp=2, tfluct_solver=1, mthbc=(2, 2, 2, 2), efix=0):
    """2-D shallow-water radial dam break on [-2.5,2.5]^2: h = 2 inside r < 0.5,
    1 outside (cell-centre test), hu = hv = 0, seeded N(0, noise) on h."""
    lo, hi = -2.5, 2.5
    d = (hi - lo) / n
    xc = lo + (np.arange(n) + 0.5) * d
    X, Y = np.meshgrid(xc, xc, indexing="xy")   # [j, i]
    h = np.where(X ** 2 + Y ** 2 < 0.25, 2.0, 1.0)
    if noise:
        h = h + noise * np.random.default_rng(seed).standard_normal(h.shape)
    q = np.zeros((3, n + 6, n + 6))
    q[0, 3:-3, 3:-3] = h
    kw = dict(mx=n, my=n, dx=d, dy=d, xlower=lo, ylower=lo, mthbc=mthbc, char_decomp=char_decomp,
              tfluct_solver=tfluct_solver, efix=efix)
    po = O.make_params(ndim=2, meqn=3, mwaves=3, rp=O.RP_SW2D, grav=1.0, **kw)
    ps = S.ClawParams(rp=S.RP_SW2D, grav=1.0, **kw)
    return po, ps, q, None


def acoustics2d(n=40, seed=5, char_decomp=0, tfluct_solver=1, mthbc=(2, 2, 2, 2), background=0.0):
    """2-D variable-coefficient acoustics on [0,1]^2: rho, K log-normal,
    smoothed; aux = (Z = sqrt(rho K), c = sqrt(K/rho)); p0 = Gaussian bumps
    plus `background` * cos(2 pi x) cos(2 pi y)."""
    rng = np.random.default_rng(seed)
    d = 1.0 / n
    ln_rho = rng.normal(0, 0.3, (n + 6, n + 6))
    ln_k = rng.normal(0, 0.3, (n + 6, n + 6))
    ker = np.exp(-0.5 * (np.arange(-6, 7) / 2.0) ** 2)
    ker /= ker.sum()
    for a in (ln_rho, ln_k):
        for ax in (0, 1):
            a[...] = np.apply_along_axis(lambda v: np.convolve(v, ker, mode="same"), ax, a)
    rho, K = np.exp(ln_rho), np.exp(ln_k)
    aux = np.stack([np.sqrt(rho * K), np.sqrt(K / rho)])
    xc = (np.arange(-3, n + 3) + 0.5) * d
    X, Y = np.meshgrid(xc, xc, indexing="xy")
    p = np.zeros_like(X)
    for _ in range(3):
        cx, cy = rng.uniform(0.2, 0.8, 2)
        p += np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * 0.05 ** 2))
    p += background * np.cos(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    q = np.zeros((3, n + 6, n + 6))
    q[0] = p
    kw = dict(mx=n, my=n, dx=d, dy=d, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=tfluct_solver)
    po = O.make_params(ndim=2, meqn=3, mwaves=2, maux=2, rp=O.RP_ACOUSTICS2D, **kw)
    ps = S.ClawParams(rp=S.RP_ACOUSTICS2D, **kw)
    return po, ps, q, aux


def with_capacity(case, seed=11):
    """Append a capacity field kappa in [0.7, 1.3] (seeded) to a case's aux and
    point mcapa at it: dtdx = dt/(dx*kappa) as flux1.f90:57-58 computes it."""
    po, ps, q, aux = case
    kappa = 1.0 + 0.3 * np.random.default_rng(seed).uniform(-1.0, 1.0, q.shape[1:])
    aux2 = kappa[None] if aux is None else np.concatenate([aux, kappa[None]])
    m = aux2.shape[0]
    po.maux, po.mcapa = m, m
    ps.maux, ps.mcapa = m, m
    return po, ps, q, np.ascontiguousarray(aux2)


def with_tvd(case, mthlim=(1, 1, 1, 1), char_decomp=0):
    """Switch a case to the second-order TVD reconstructions (lim_type = 1,
    reconstruct.f90:525-761) with the given limiters per component / field /
    wave and char_decomp (0 tvd2, 1 tvd2_wave, 2 tvd2_char)."""
    po, ps, q, aux = case
    po.lim_type = ps.lim_type = 1
    po.char_decomp = ps.char_decomp = char_decomp
    for k in range(4):
        po.mthlim[k] = int(mthlim[k])
    ps.mthlim = tuple(int(v) for v in mthlim)
    return po, ps, q, aux


def with_poly(case, char_decomp=0):
    """Switch a case to the unlimited polynomial reconstruction of order 3
    (lim_type = 0, polyrecon.f90: 0 q2qlqr_poly, 1 q2qlqr_poly_wave)."""
    po, ps, q, aux = case
    po.lim_type = ps.lim_type = 0
    po.char_decomp = ps.char_decomp = char_decomp
    po.mthlim[0] = 3
    ps.mthlim = (3,) + tuple(ps.mthlim[1:])
    return po, ps, q, aux


def swirl(n=40, tperiod=0.0, char_decomp=0):
    """apps/advection/2d/swirl: [0,1]^2, extrapolation bc, edge velocities
    from the stream function psi = sin^2(pi x) sin^2(pi y)/pi (setaux.f,
    ghost cells included), q = 1 for x < 0.5 else 0 (qinit.f90), WENO5, the
    swapped second solve (tfluct_solver 0); b4step scales the velocities by
    cos(2 pi (t + dt/2)/tperiod) when tperiod > 0."""
    d = 1.0 / n
    pi = 4.0 * np.arctan(1.0)
    psi = lambda x, y: (np.sin(pi * x) * np.sin(pi * x)) * (np.sin(pi * y) * np.sin(pi * y)) / pi
    idx = np.arange(-2, n + 4)                       # cells 1-mbc .. n+mbc
    XL, YL = np.meshgrid((idx - 1) * d, (idx - 1) * d, indexing="xy")
    aux = np.stack([-(psi(XL, YL + d) - psi(XL, YL)) / d, (psi(XL + d, YL) - psi(XL, YL)) / d])
    q = np.zeros((1, n + 6, n + 6))
    xc = (np.arange(1, n + 1) - 0.5) * d
    q[0, 3:-3, 3:-3] = np.where(xc[None, :] < 0.5, 1.0, 0.0) * np.ones((n, 1))
    kw = dict(mx=n, my=n, dx=d, dy=d, mthbc=(1, 1, 1, 1), char_decomp=char_decomp, tfluct_solver=0)
    po = O.make_params(ndim=2, meqn=1, mwaves=1, maux=2, rp=O.RP_ADVECTION2D, **kw)
    po.b4step = 1 if tperiod > 0 else 0
    po.tperiod = tperiod
    ps = S.ClawParams(rp=S.RP_ADVECTION2D, **kw)
    return po, ps, q, np.ascontiguousarray(aux)


def radial_sw(mx=200, char_decomp=0, tfluct_solver=0, src=True, efix=1):
    """Radially symmetric dam break, apps/shallowWater/2dRadialDam/
    1dRadialSymm-qwave: r in [0, 2.5], h = 2 for r < 0.5 else 1, hu = 0,
    g = 1, wall at r = 0 and extrapolation outside, rp1sw.f + the radial
    source term of its src1.f90."""
    dx = 2.5 / mx
    xc = (np.arange(mx) + 0.5) * dx
    q = np.zeros((2, mx + 6))
    q[0, 3:-3] = np.where(xc < 0.5, 2.0, 1.0)
    kw = dict(mx=mx, dx=dx, xlower=0.0, mthbc=(3, 1), char_decomp=char_decomp, tfluct_solver=tfluct_solver,
              grav=1.0, efix=efix)
    po = O.make_params(meqn=2, mwaves=2, rp=O.RP_SW1D, src_term=O.SRC_RADIAL_SW if src else O.SRC_NONE, **kw)
    ps = S.ClawParams(rp=S.RP_SW1D, src_term=S.SRC_RADIAL_SW if src else S.SRC_NONE, **kw)
    return po, ps, q, None


def bathymetry_sw(mx=200, eps=0.2, char_decomp=0, tfluct_solver=1):
    """Perturbation of a lake at rest over a bump, apps/shallowWater/
    1dPerturbSteady (setaux.f90, qinit.f90, setprob g = 9.81, eps = 0.2) on
    [0, 2] with extrapolation bc, solved with rp1sw.f and the bathymetry
    source of that app's src1.f90 (b in aux(:,1))."""
    dx = 2.0 / mx
    xa = (np.arange(-3, mx + 3) + 0.5) * dx
    b = np.where((xa >= 1.4) & (xa <= 1.6), 0.25 * (np.cos(10 * np.pi * (xa - 1.5)) + 1.0), 0.0)
    aux = b[None, :].copy()
    q = np.zeros((2, mx + 6))
    xc = xa[3:-3]
    q[0, 3:-3] = 1.0 - b[3:-3] + np.where((xc >= 1.1) & (xc <= 1.2), eps, 0.0)
    kw = dict(mx=mx, dx=dx, xlower=0.0, mthbc=(1, 1), char_decomp=char_decomp, tfluct_solver=tfluct_solver,
              grav=9.81, maux=1)
    po = O.make_params(meqn=2, mwaves=2, rp=O.RP_SW1D, src_term=O.SRC_BATHYMETRY_SW, **kw)
    ps = S.ClawParams(rp=S.RP_SW1D, src_term=S.SRC_BATHYMETRY_SW, **kw)
    return po, ps, q, aux


def fwave_bathymetry(mx=200, eps=0.2, char_decomp=0, tfluct_solver=1):
    """apps/shallowWater/1dPerturbSteady as the app runs it: the f-wave solver
    (rpf-wave.f90) with the bathymetry source inside its tfluct
    (tfluctf-wave.f90), the library's zero src; data as bathymetry_sw."""
    po, ps, q, aux = bathymetry_sw(mx=mx, eps=eps, char_decomp=char_decomp, tfluct_solver=tfluct_solver)
    po.rp, po.src_term = O.RP_SWF_BATHY, O.SRC_NONE
    ps.rp, ps.src_term = S.RP_SWF_BATHY, S.SRC_NONE
    return po, ps, q, aux


def fwave_radial(mx=200, kappa=False, char_decomp=0, tfluct_solver=1):
    """The radial dam break of radial_sw with the f-wave solvers of
    2dRadialDam/1dRadialSymm-fwave (aux = (r, dx), setaux.f90) or, with
    kappa, 1dRadialSymm-fwave-kappa (aux = (r(i-1/2), r, r, dx), capacity
    aux(:,2))."""
    dx = 2.5 / mx
    xa = (np.arange(-3, mx + 3) + 0.5) * dx
    if kappa:
        xi = np.arange(-3, mx + 3) * dx
        aux = np.ascontiguousarray(np.stack([xi, xa, xa, np.full_like(xa, dx)]))
        rp_o, rp_s, mcapa = O.RP_SWF_KAPPA, S.RP_SWF_KAPPA, 2
    else:
        aux = np.ascontiguousarray(np.stack([xa, np.full_like(xa, dx)]))
        rp_o, rp_s, mcapa = O.RP_SWF_RADIAL, S.RP_SWF_RADIAL, 0
    q = np.zeros((2, mx + 6))
    q[0, 3:-3] = np.where(xa[3:-3] < 0.5, 2.0, 1.0)
    kw = dict(mx=mx, dx=dx, xlower=0.0, mthbc=(3, 1), char_decomp=char_decomp, tfluct_solver=tfluct_solver,
              grav=1.0, maux=aux.shape[0], mcapa=mcapa)
    po = O.make_params(meqn=2, mwaves=2, rp=rp_o, **kw)
    ps = S.ClawParams(rp=rp_s, **kw)
    return po, ps, q, aux


def acoustics_const(mx=200, rho=1.0, bulk=4.0, mthbc=(3, 3), char_decomp=0, tfluct_solver=0, smooth=False):
    """apps/acoustics/1d/homogeneous (setrun.py: [-1, 1], walls, rho 1, bulk
    4): p0 = exp(-50 (x-0.3)^2) cos(20 (x-0.3)) for x <= 0.3 (qinit.f), u0 = 0;
    smooth: the Gaussian alone, for the exact-solution check."""
    dx = 2.0 / mx
    xc = -1.0 + (np.arange(mx) + 0.5) * dx
    p0 = np.exp(-50.0 * (xc - 0.3) ** 2)
    if not smooth:
        p0 = np.where(xc > 0.3, 0.0, p0 * np.cos(20.0 * (xc - 0.3)))
    q = np.zeros((2, mx + 6))
    q[0, 3:-3] = p0
    kw = dict(mx=mx, dx=dx, xlower=-1.0, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=tfluct_solver,
              rho=rho, bulk=bulk)
    po = O.make_params(meqn=2, mwaves=2, rp=O.RP_ACOUSTICS_CONST, **kw)
    ps = S.ClawParams(rp=S.RP_ACOUSTICS_CONST, **kw)
    return po, ps, q, None


def acoustics_fwave(mx=200, char_decomp=2, tfluct_solver=1, mthbc=(1, 1)):
    """apps/acoustics/1d/fwave: the interface problem of acoustics1d in strain
    / momentum form, q = (eps, rho u) with eps = -p/bulk, aux = (rho, bulk)."""
    from acoustics_exact import InterfaceProblem
    ap = InterfaceProblem()
    dx = 20.0 / mx
    za = ap.setaux(mx)                      # (Z, c)
    rho, bulk = za[0] / za[1], za[0] * za[1]
    aux = np.ascontiguousarray(np.stack([rho, bulk]))
    qp = ap.qinit(mx, za)                   # (p, u)
    q = np.stack([-qp[0] / bulk, rho * qp[1]])
    kw = dict(mx=mx, dx=dx, xlower=-10.0, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=tfluct_solver)
    po = O.make_params(meqn=2, mwaves=2, maux=2, rp=O.RP_ACOUSTICS_FWAVE, **kw)
    ps = S.ClawParams(rp=S.RP_ACOUSTICS_FWAVE, **kw)
    return po, ps, q, aux


def traffic(mx=300, rho=(0.13, 0.1), umax=(2.0, 1.0), lower=-20.0, upper=40.0, mthbc=(1, 1), char_decomp=0,
            tfluct_solver=1):
    """apps/traffic/congTraffic (setrun.py: [-20, 40], densities 0.13 / 0.1,
    speed limits 2 / 1 on either side of x = 0, extrapolation bc): q = density,
    aux = umax per cell (the app's setaux.f90 leaves aux unset; the limits of
    its setprob data are used, split at x = 0 like its qinit)."""
    dx = (upper - lower) / mx
    xa = lower + (np.arange(-3, mx + 3) + 0.5) * dx
    aux = np.ascontiguousarray(np.where(xa < 0.0, umax[0], umax[1])[None, :])
    q = np.zeros((1, mx + 6))
    q[0, 3:-3] = np.where(xa[3:-3] < 0.0, rho[0], rho[1])
    kw = dict(mx=mx, dx=dx, xlower=lower, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=tfluct_solver)
    po = O.make_params(meqn=1, mwaves=1, maux=1, rp=O.RP_TRAFFIC, **kw)
    ps = S.ClawParams(rp=S.RP_TRAFFIC, **kw)
    return po, ps, q, aux


def advection_cons(mx=300, u=(2.0, 1.0), rho=(0.3333, 0.1), lower=-45.0, upper=45.0, mthbc=(1, 1),
                   char_decomp=0):
    """apps/traffic/flux-uq: (u(x) q)_x = 0 with cell velocities u1 / u2 and
    densities rho1 / rho2 on either side of x = 0 (setaux.f90, qinit.f90),
    [-45, 45], extrapolation bc, the swapped second solve."""
    dx = (upper - lower) / mx
    xa = lower + (np.arange(-3, mx + 3) + 0.5) * dx
    aux = np.ascontiguousarray(np.where(xa < 0.0, u[0], u[1])[None, :])
    q = np.zeros((1, mx + 6))
    q[0, 3:-3] = np.where(xa[3:-3] < 0.0, rho[0], rho[1])
    kw = dict(mx=mx, dx=dx, xlower=lower, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=0)
    po = O.make_params(meqn=1, mwaves=1, maux=1, rp=O.RP_ADVECTION_CONS, **kw)
    ps = S.ClawParams(rp=S.RP_ADVECTION_CONS, **kw)
    return po, ps, q, aux


def stegoton(mx=200, char_decomp=0, tfluct_solver=1, mthbc=(1, 1), amp=0.05):
    """apps/elasticity/stegoton: layered medium (setaux.f: rho, K = 1, 1 in
    the first half of each unit cell, 4, 4 in the second; aux(:,3) = 0, so the
    stress is exp(K eps) - 1), strain eps and momentum rho u; a smooth strain
    pulse stands in for the app's moving-wall boundary condition (mthbc 0,
    user code that the device path does not run)."""
    lower, upper = 0.0, 30.0
    dx = (upper - lower) / mx
    xa = lower + (np.arange(-3, mx + 3) + 0.5) * dx
    frac = xa - np.trunc(xa)     # setaux.f: ix = xcell truncates toward zero
    rho = np.where(frac < 0.5, 1.0, 4.0)
    K = np.where(frac < 0.5, 1.0, 4.0)
    aux = np.ascontiguousarray(np.stack([rho, K, np.zeros_like(xa)]))
    q = np.zeros((2, mx + 6))
    q[0, 3:-3] = amp * np.exp(-((xa[3:-3] - 8.0) / 2.0) ** 2)
    kw = dict(mx=mx, dx=dx, xlower=lower, mthbc=mthbc, char_decomp=char_decomp, tfluct_solver=tfluct_solver)
    po = O.make_params(meqn=2, mwaves=2, maux=3, rp=O.RP_STEGOTON, **kw)
    ps = S.ClawParams(rp=S.RP_STEGOTON, **kw)
    return po, ps, q, aux


def oracle_riemann_window(job):
    """Process-pool worker: the oracle's sharpclaw() on one 1-D Euler Riemann
    instance of the batched workload (Roe + entropy fix, componentwise WENO5,
    tfluct_solver 0, SSPRK(3,3), extrapolation bc) over [0, tend].  job =
    (mx, dx, q, dt_initial, tend, (cfl_max, cfl_desired)); returns the final q
    and the run's outputs as a dict."""
    mx, dx, q, dt0, tend, (cfl_max, cfl_desired) = job
    po = O.make_params(mx=mx, meqn=3, mwaves=3, dx=dx, rp=O.RP_EULER, gamma=1.4, mthbc=(1, 1),
                       char_decomp=0, tfluct_solver=0)
    qo, ro = O.sharpclaw(po, q, None, tstart=0.0, tend=tend, dt_initial=dt0, cfl_max=cfl_max,
                         cfl_desired=cfl_desired, time_integrator=3)
    return qo, dict(steps_taken=ro.steps_taken, rejected=ro.rejected, info=ro.info, tend=ro.tend,
                    dt_last=ro.dt_last, cfl_maxused=ro.cfl_maxused)
