"""The hand-written adjoint (scl_adjoint_step, sharpclaw_b200.adjoint) on a GPU,
for each integrator (SSPRK(2,2), (4,2), (3,3), (10,4)) with componentwise
WENO5 and, for SSPRK(3,3) and (10,4), characteristic-wise WENO5, on 2-D
variable-coefficient acoustics and on the 1-D interface app
(apps/acoustics/1d/interface, periodic):

* one step: the forward step of the FP64_STRICT solver equals the
  FP64 PyTorch restatement (tests/torch_ref.py, same evaluation order) bit for
  bit, and the vector-Jacobian product equals torch.autograd through that
  restatement to 1e-11 relative;
* the dot-product identity <J v, w> = <v, J^T w>;
* the gradient of the misfit through 60 steps with checkpoints every 20
  matches central finite differences along random directions to 1e-4
  (and torch.autograd through 60 steps of the restatement to ~1e-12).

The same states must enter both sides: where cell differences are ~1e-18 the
smoothness indicators are ~epsilon = 1e-36 and the WENO weights' derivatives
amplify state differences by ~1e6, so a forward that rounds differently (FMA)
gives a different -- equally valid -- linearisation there.  The
finite-difference check therefore uses initial data with a smooth background,
which keeps every cell away from that regime.
"""
import numpy as np
import pytest
import torch

import cases
import torch_ref
import sharpclaw_b200 as S
from sharpclaw_b200 import adjoint as A

pytestmark = pytest.mark.gpu


def _problem(n=24, seed=5, background=0.0, ti=3, cd=0):
    po, ps, q, aux = cases.acoustics2d(n=n, seed=seed, background=background, char_decomp=cd)
    # periodic aux: ghost cells are the images of interior cells
    inner = aux[:, 3:-3, 3:-3]
    aux = np.ascontiguousarray(np.pad(inner, ((0, 0), (3, 3), (3, 3)), mode="wrap"))
    ps.time_integrator = ti
    dt = {1: 0.4, 2: 0.8, 3: 0.4, 4: 1.2}[ti] * ps.dx / float(aux[1].max())
    return ps, q, aux, dt


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _cpu(a):
    # the PyTorch restatement runs on the CPU: its elementwise ops are then
    # plain IEEE operations in the Fortran order, bit-identical to the oracle
    return torch.from_numpy(np.ascontiguousarray(a))


@pytest.mark.parametrize("ti,cd", [(1, 0), (2, 0), (3, 0), (4, 0), (3, 2), (4, 2)])
def test_forward_step_matches_torch_restatement(ti, cd):
    ps, q, aux, dt = _problem(ti=ti, cd=cd)
    with S.Solver(ps, "fp64_strict") as s:
        s.set_aux(aux)
        s.set_q(q)
        s.rk_step(dt)
        got = s.get_q()[:, 3:-3, 3:-3]
    Z, c = _cpu(aux[0, 3:-3, 3:-3]), _cpu(aux[1, 3:-3, 3:-3])
    ref = torch_ref.rk(ti)(_cpu(q[:, 3:-3, 3:-3]), Z, c, dt, ps.dx, ps.dy, cd).numpy()
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("ti,cd", [(1, 0), (2, 0), (3, 0), (4, 0), (3, 2), (4, 2)])
def test_adjoint_step_matches_autograd(ti, cd):
    ps, q, aux, dt = _problem(ti=ti, cd=cd)
    rng = np.random.default_rng(1)
    lam = np.zeros_like(q)
    lam[:, 3:-3, 3:-3] = rng.standard_normal(lam[:, 3:-3, 3:-3].shape)
    with S.Solver(ps, "fp64_strict") as s:
        s.set_aux(aux)
        got = A.adjoint_step(s, _dev(q), _dev(lam), dt).cpu().numpy()[:, 3:-3, 3:-3]
    Z, c = _cpu(aux[0, 3:-3, 3:-3]), _cpu(aux[1, 3:-3, 3:-3])
    x = _cpu(q[:, 3:-3, 3:-3]).requires_grad_(True)
    y = torch_ref.rk(ti)(x, Z, c, dt, ps.dx, ps.dy, cd)
    (g,) = torch.autograd.grad(y, x, _cpu(lam[:, 3:-3, 3:-3]))
    ref = g.numpy()
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("ti,cd", [(1, 0), (2, 0), (3, 0), (4, 0), (3, 2), (4, 2)])
def test_adjoint_dot_product_identity(ti, cd):
    ps, q, aux, dt = _problem(n=20, seed=8, ti=ti, cd=cd)
    rng = np.random.default_rng(2)
    w = np.zeros_like(q)
    w[:, 3:-3, 3:-3] = rng.standard_normal(w[:, 3:-3, 3:-3].shape)
    v = rng.standard_normal(q[:, 3:-3, 3:-3].shape)
    Z, c = _cpu(aux[0, 3:-3, 3:-3]), _cpu(aux[1, 3:-3, 3:-3])
    x = _cpu(q[:, 3:-3, 3:-3])
    _, jv = torch.func.jvp(lambda t: torch_ref.rk(ti)(t, Z, c, dt, ps.dx, ps.dy, cd), (x,), (_cpu(v),))
    with S.Solver(ps, "fp64_strict") as s:
        s.set_aux(aux)
        jtw = A.adjoint_step(s, _dev(q), _dev(w), dt).cpu().numpy()[:, 3:-3, 3:-3]
    lhs = float((jv.cpu().numpy() * w[:, 3:-3, 3:-3]).sum())
    rhs = float((v * jtw).sum())
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("ti,cd", [(1, 0), (2, 0), (3, 0), (4, 0), (3, 2), (4, 2)])
def test_misfit_gradient_against_finite_differences(ti, cd):
    ps, q, aux, dt = _problem(n=32, seed=3, background=0.05, ti=ti, cd=cd)
    nsteps = {1: 60, 2: 30, 3: 60, 4: 20}[ti]
    rng = np.random.default_rng(4)
    p_obs = _dev(q[0, 3:-3, 3:-3] * 0.9 + 0.01 * rng.standard_normal(q[0, 3:-3, 3:-3].shape))
    with S.Solver(ps, "fp64") as s:
        s.set_aux(aux)
        p0 = _dev(q[0, 3:-3, 3:-3]).requires_grad_(True)
        J = A.wave_misfit(p0, s, dt, nsteps, p_obs, checkpoint_every=20)
        (g,) = torch.autograd.grad(J, p0)
        for k in range(3):
            d = _dev(rng.standard_normal(q[0, 3:-3, 3:-3].shape))
            # white-noise directions excite the WENO nonlinearity: central
            # differences converge as O(h^2) with a large constant (1.7e-4 at
            # h = 1e-6, 1.7e-6 at h = 1e-7 for this problem)
            h = 1e-7
            Jp = A.wave_misfit(p0.detach() + h * d, s, dt, nsteps, p_obs)
            Jm = A.wave_misfit(p0.detach() - h * d, s, dt, nsteps, p_obs)
            fd = float((Jp - Jm) / (2 * h))
            ad = float((g * d).sum())
            assert abs(fd - ad) <= 1e-4 * abs(fd), (k, fd, ad)


# ---- 1-D: the acoustics interface app (apps/acoustics/1d/interface), periodic ----

def _problem1d(mx=120, ti=3, cd=0, background=0.0):
    po, ps, q, aux = cases.acoustics1d(mx=mx, char_decomp=cd, mthbc=(2, 2))
    aux = np.ascontiguousarray(np.pad(aux[:, 3:-3], ((0, 0), (3, 3)), mode="wrap"))
    # a smooth periodic background keeps every cell difference well above
    # rounding, out of the epsilon regime of the smoothness indicators
    q = q.copy()
    x = ps.xlower + (np.arange(mx) + 0.5) * ps.dx
    q[0, 3:-3] += background * np.cos(2 * np.pi * (x - ps.xlower) / (mx * ps.dx) + 0.3)
    ps.time_integrator = ti
    dt = {1: 0.4, 2: 0.8, 3: 0.4, 4: 1.2}[ti] * ps.dx / float(aux[1].max())
    return ps, q, aux, dt


CASES_1D = [(1, 0), (3, 0), (4, 0), (3, 2), (4, 2)]


@pytest.mark.parametrize("ti,cd", CASES_1D)
def test_1d_forward_step_matches_torch_restatement(ti, cd):
    ps, q, aux, dt = _problem1d(ti=ti, cd=cd)
    with S.Solver(ps, "fp64_strict") as s:
        s.set_aux(aux)
        s.set_q(q)
        s.rk_step(dt)
        got = s.get_q()[:, 3:-3]
    Z, c = _cpu(aux[0, 3:-3]), _cpu(aux[1, 3:-3])
    ref = torch_ref.rk(ti)(_cpu(q[:, 3:-3]), Z, c, dt, ps.dx, ps.dx, cd).numpy()
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("ti,cd", CASES_1D)
def test_1d_adjoint_step_matches_autograd_and_dot_product(ti, cd):
    ps, q, aux, dt = _problem1d(ti=ti, cd=cd)
    rng = np.random.default_rng(6)
    lam = np.zeros_like(q)
    lam[:, 3:-3] = rng.standard_normal(lam[:, 3:-3].shape)
    v = rng.standard_normal(q[:, 3:-3].shape)
    with S.Solver(ps, "fp64_strict") as s:
        s.set_aux(aux)
        got = A.adjoint_step(s, _dev(q), _dev(lam), dt).cpu().numpy()[:, 3:-3]
    Z, c = _cpu(aux[0, 3:-3]), _cpu(aux[1, 3:-3])
    f = lambda t: torch_ref.rk(ti)(t, Z, c, dt, ps.dx, ps.dx, cd)
    x = _cpu(q[:, 3:-3]).requires_grad_(True)
    (g,) = torch.autograd.grad(f(x), x, _cpu(lam[:, 3:-3]))
    ref = g.numpy()
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
    _, jv = torch.func.jvp(f, (_cpu(q[:, 3:-3]),), (_cpu(v),))
    lhs = float((jv.numpy() * lam[:, 3:-3]).sum())
    rhs = float((v * got).sum())
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("ti,cd", [(3, 0), (4, 2)])
def test_1d_misfit_gradient_against_autograd_and_finite_differences(ti, cd):
    ps, q, aux, dt = _problem1d(mx=200, ti=ti, cd=cd, background=0.05)
    nsteps = 40
    rng = np.random.default_rng(7)
    p_obs = q[0, 3:-3] * 0.9 + 0.01 * rng.standard_normal(q[0, 3:-3].shape)
    Z, c = _cpu(aux[0, 3:-3]), _cpu(aux[1, 3:-3])

    def J_ref(p0):
        y = torch.stack([p0, torch.zeros_like(p0)])
        for _ in range(nsteps):
            y = torch_ref.rk(ti)(y, Z, c, dt, ps.dx, ps.dx, cd)
        return 0.5 * ((y[0] - _cpu(p_obs)) ** 2).sum()

    x = _cpu(q[0, 3:-3]).requires_grad_(True)
    (g_ref,) = torch.autograd.grad(J_ref(x), x)
    with S.Solver(ps, "fp64") as s:
        s.set_aux(aux)
        p0 = _dev(q[0, 3:-3]).requires_grad_(True)
        J = A.wave_misfit(p0, s, dt, nsteps, _dev(p_obs), checkpoint_every=15)
        (g,) = torch.autograd.grad(J, p0)
        g_cpu = g.cpu().numpy()
        assert np.abs(g_cpu - g_ref.numpy()).max() <= 1e-9 * np.abs(g_ref.numpy()).max()
        for k in range(3):
            d = _dev(rng.standard_normal(q[0, 3:-3].shape))
            # the pulse crossing the impedance jump keeps the WENO weights
            # switching: central differences of this misfit converge slowly in
            # h (3e-4 at h = 1e-7, 4e-6 at h = 1e-8 along a white-noise
            # direction), so h = 1e-8, where rounding (1e-16 J / h) is still small
            h = 1e-8
            Jp = A.wave_misfit(p0.detach() + h * d, s, dt, nsteps, _dev(p_obs))
            Jm = A.wave_misfit(p0.detach() - h * d, s, dt, nsteps, _dev(p_obs))
            fd = float((Jp - Jm) / (2 * h))
            ad = float((g * d).sum())
            assert abs(fd - ad) <= 1e-4 * abs(fd), (k, fd, ad)
