"""Exact solution of the 1-D acoustics interface problem (known-answer test).

Restates, in Python 3, the characteristic-tracing solution of
apps/acoustics/1d/interface/actools.py (AcousticsProblem: impedances z=rho*c,
transmission CT_lr = 2 z1/(z0+z1), reflection CR_lr = (z1-z0)/(z0+z1), pressure
p = w1+w2, velocity u = (w2-w1)/z) for a single material interface at x = 0
and a right-going initial pulse that meets the interface once before the final
time, and the initial data / medium setup of the reference app
(qinit.f ic=9 'C5 Newton polynomial' cell averages, setaux.f90 cell
assignment by right cell edge).  sharpclawtest.py compares numerical cell
averages with exact cell averages in the 1-norm; tests here do the same.
"""
import numpy as np


class InterfaceProblem:
    def __init__(self, rho=(1.0, 4.0), c=(1.0, 0.5), a=1.0, x0=-4.0, xlower=-10.0,
                 xupper=10.0, interface=0.0):
        self.rho = np.asarray(rho, float)
        self.c = np.asarray(c, float)
        self.z = self.rho * self.c
        self.a, self.x0 = a, x0
        self.xlower, self.xupper, self.xi = xlower, xupper, interface
        z0, z1 = self.z
        self.CT = 2.0 * z1 / (z0 + z1)          # actools.py:82
        self.CR = (z1 - z0) / (z0 + z1)         # actools.py:83

    def p0(self, y):
        """initial pressure: (y-x0-a)^6 (y-x0+a)^6 / a^12 on |y-x0|<=a (actools.py q0)."""
        y = np.asarray(y, float)
        r = y - self.x0
        out = (r - self.a) ** 6 * (r + self.a) ** 6 / self.a ** 12
        return np.where(np.abs(r) <= self.a, out, 0.0)

    def pu(self, x, t):
        """pressure and velocity at points x, time t (one interface crossing)."""
        x = np.asarray(x, float)
        c0, c1 = self.c
        z0, z1 = self.z
        left = x < self.xi
        xr = x - self.xi
        p_inc = self.p0(x - c0 * t)
        p_ref = self.CR * self.p0(self.xi - c0 * (t + xr / c0))
        p_tr = self.CT * self.p0(self.xi - c0 * (t - xr / c1))
        p = np.where(left, p_inc + p_ref, p_tr)
        u = np.where(left, (p_inc - p_ref) / z0, p_tr / z1)
        return p, u

    def cell_averages(self, mx, t, nq=10):
        dx = (self.xupper - self.xlower) / mx
        xe = self.xlower + dx * np.arange(mx + 1)
        g, w = np.polynomial.legendre.leggauss(nq)
        pts = 0.5 * (xe[:-1, None] + xe[1:, None]) + 0.5 * dx * g[None, :]
        p, u = self.pu(pts, t)
        return (p * w).sum(1) * 0.5, (u * w).sum(1) * 0.5

    def setaux(self, mx, mbc=3):
        """setaux.f90:229-237: material by right cell edge xlower+i*dx > interface."""
        dx = (self.xupper - self.xlower) / mx
        i = np.arange(1 - mbc, mx + mbc + 1)
        mat = (self.xlower + i * dx > self.xi).astype(int)
        aux = np.zeros((2, mx + 2 * mbc))
        aux[0] = self.rho[mat] * self.c[mat]
        aux[1] = self.c[mat]
        return aux

    def qinit(self, mx, aux, mbc=3):
        """qinit.f:152-175 (ic=9): exact cell averages of the C5 pulse, zeroed
        where the cell centre lies outside the support; u = p / Z."""
        dx = (self.xupper - self.xlower) / mx
        a, x0 = self.a, self.x0
        xc = self.xlower + (np.arange(1, mx + 1) - 0.5) * dx

        def F(x):
            return (x ** 13 / (13.0 * a ** 12) - 6.0 * x ** 11 / (11.0 * a ** 10)
                    + 5.0 * x ** 9 / (3.0 * a ** 8) - 20.0 * x ** 7 / (7.0 * a ** 6)
                    + 3.0 * x ** 5 / a ** 4 - 2.0 * x ** 3 / (a * a) + x)

        p = (F(xc + 0.5 * dx - x0) - F(xc - 0.5 * dx - x0)) / dx
        p = np.where(np.abs(xc - x0) > a, 0.0, p)
        q = np.zeros((2, mx + 2 * mbc))
        q[0, mbc:-mbc] = p
        q[1, mbc:-mbc] = p / aux[0, mbc:-mbc]
        return q
