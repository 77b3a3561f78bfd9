"""Plain PyTorch FP64 restatement of the 2-D acoustics WENO step (periodic).

Used as the floating-point reference of the adjoint: torch.autograd through
this restatement gives the exact vector-Jacobian product of the same
discrete operator -- dq = dt*L(q) of src/2d/flux2.f90 with componentwise
weno5 (src/reconstruct.f90:77-143), the acoustics Riemann solver
(apps/acoustics/1d/interface/rp1acv.f:49-80 applied normal to each sweep)
and tfluct (tfluct1acv.f:134-166) -- and SSPRK(3,3) (src/sharpclaw.f90:337-376).
Arrays are interior cells only, (3, ny, nx); periodic bc are rolls.
"""
import numpy as np
import torch

EPS = float(np.float32(1e-36))


def weno_side(dm2, dm1, d0, dp1, im):
    t1 = im * (dm2 - dm1)
    t2 = im * (dm1 - d0)
    t3 = im * (d0 - dp1)
    # 13.*t**2 + 3.*x**2 associated as the Fortran source (reconstruct.f90:117-119)
    x1, x2, x3 = dm2 - 3.0 * dm1, dm1 + d0, 3.0 * d0 - dp1
    tt1 = (EPS + (13.0 * (t1 * t1) + 3.0 * (x1 * x1))) ** 2
    tt2 = (EPS + (13.0 * (t2 * t2) + 3.0 * (x2 * x2))) ** 2
    tt3 = (EPS + (13.0 * (t3 * t3) + 3.0 * (x3 * x3))) ** 2
    s1 = tt2 * tt3
    s2 = 6.0 * tt1 * tt3
    s3 = 3.0 * tt1 * tt2
    t0 = 1.0 / ((s1 + s2) + s3)
    s1 = s1 * t0
    s3 = s3 * t0
    return ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) / 3.0


def sweep(q, Z, c, dtdx, axis, mu, cd=0):
    r = lambda a, s: torch.roll(a, s, dims=axis)   # r(a, 1)[i] = a[i-1]
    if cd == 2:
        qr, ql = char_edges(q, Z, axis, mu)
    else:
        d = q - r(q, 1)
        D0, D1, D2, D3 = r(d, 1), d, r(d, -1), r(d, -2)
        qr = weno_side(D0, D1, D2, D3, 1.0) + (-r(q, 1) + 7.0 * (q + r(q, -1)) - r(q, -2)) / 12.0
        ql = weno_side(D3, D2, D1, D0, -1.0) + (-r(q, 2) + 7.0 * (r(q, 1) + q) - r(q, -1)) / 12.0
    dl = ql - r(qr, 1)                      # interface i: ql(i) - qr(i-1)
    zi, zim = Z, r(Z, 1)
    a1 = (-dl[0] + zi * dl[mu]) / (zim + zi)
    a2 = (dl[0] + zim * dl[mu]) / (zim + zi)
    s1, s2 = -r(c, 1), c
    zero = torch.zeros_like(a1)
    M = q.shape[0]
    w1 = [-a1 * zim] + [zero] * (M - 1)
    w1[mu] = a1
    w2 = [a2 * zi] + [zero] * (M - 1)
    w2[mu] = a2
    amdq = torch.stack([s1 * w for w in w1])
    apdq = torch.stack([s2 * w for w in w2])
    dt_ = qr - ql                           # tfluct: left ql(i), right qr(i), aux of cell i
    b1 = (-dt_[0] + Z * dt_[mu]) / (2.0 * Z)
    b2 = (dt_[0] + Z * dt_[mu]) / (2.0 * Z)
    v1 = [-b1 * Z] + [zero] * (M - 1)
    v1[mu] = b1
    v2 = [b2 * Z] + [zero] * (M - 1)
    v2[mu] = b2
    adq = torch.stack([-c * a + c * b for a, b in zip(v1, v2)])
    amdq_next = torch.roll(amdq, -1, dims=axis)
    return -dtdx * (apdq + adq + amdq_next)


def char_edges(q, Z, axis, mu):
    """weno5_char (reconstruct.f90:146-241) with the acoustics eigenvectors of
    each interface (evec.f90:196-206 with the tangential velocity as a third,
    zero-speed field): returns qr(c) and ql(c) of every cell, accumulated in
    the kernel's order (full 3x3 sums, zero entries included)."""
    r = lambda a, s: torch.roll(a, s, dims=axis)
    M = q.shape[0]
    zim, zi = r(Z, 1), Z                    # interface i between cells i-1 and i
    z = 1.0 / (zim + zi)
    zero, one = torch.zeros_like(Z), torch.ones_like(Z)
    evl = [[zero] * M for _ in range(M)]
    evr = [[zero] * M for _ in range(M)]
    evr[0][0], evr[0][1], evr[mu][0], evr[mu][1] = -zim, zi, one, one
    evl[0][0], evl[0][mu], evl[1][0], evl[1][mu] = -1.0 * z, zi * z, 1.0 * z, zim * z
    if M == 3:
        mv = 3 - mu
        evr[mv][2], evl[2][mv] = one, one
    d = q - r(q, 1)                          # d(j) = q(j) - q(j-1)
    dk = [r(d, 2 - k) for k in range(5)]     # at interface i: d(i-2+k)
    cen = ((-r(q, 2)) + 7.0 * (r(q, 1) + q)) - r(q, -1)
    QR = [cen[m] / 12.0 for m in range(M)]   # qr(i-1)
    QL = [cen[m] / 12.0 for m in range(M)]   # ql(i)
    for p in range(M):
        h = []
        for k in range(5):
            s = torch.zeros_like(Z)
            for m in range(M):
                s = s + evl[p][m] * dk[k][m]
            h.append(s)
        u1 = weno_side(h[0], h[1], h[2], h[3], 1.0)
        u2 = weno_side(h[4], h[3], h[2], h[1], -1.0)
        for m in range(M):
            QR[m] = QR[m] + evr[m][p] * u1
            QL[m] = QL[m] + evr[m][p] * u2
    return r(torch.stack(QR), -1), torch.stack(QL)


def D(q, Z, c, dt, dx, dy, cd=0):
    if q.dim() == 2:                         # 1-D: (p, u) on one line
        return sweep(q, Z, c, dt / dx, -1, 1, cd)
    return sweep(q, Z, c, dt / dx, -1, 1, cd) + sweep(q, Z, c, dt / dy, -2, 2, cd)


def ssprk3(q, Z, c, dt, dx, dy, cd=0):
    q1 = q + D(q, Z, c, dt, dx, dy, cd)
    q2 = 0.75 * q + 0.25 * (q1 + D(q1, Z, c, dt, dx, dy, cd))
    return (q + 2.0 * (q2 + D(q2, Z, c, dt, dx, dy, cd))) / 3.0


def ssp104(q, Z, c, dt, dx, dy, cd=0):
    """ts_ssp104 (sharpclaw.f90:380-464) in the stage kernels' order."""
    def Dq(x):
        return D(x, Z, c, dt, dx, dy, cd)
    s = q
    for _ in range(4):
        s = s + (1.0 / 6.0) * Dq(s)
    r2 = s + (1.0 / 6.0) * Dq(s)
    r1 = 0.04 * q + 0.36 * r2
    s = 0.6 * q + 0.4 * r2
    for _ in range(4):
        s = s + (1.0 / 6.0) * Dq(s)
    return (r1 + 0.6 * s) + 0.1 * Dq(s)


def ssp22(q, Z, c, dt, dx, dy, cd=0):
    """ts_ssp22 (sharpclaw.f90:247-276)."""
    q1 = q + D(q, Z, c, dt, dx, dy, cd)
    return 0.5 * ((q + q1) + D(q1, Z, c, dt, dx, dy, cd))


def ssp42(q, Z, c, dt, dx, dy, cd=0):
    """ts_ssp42 (sharpclaw.f90:280-333)."""
    s = q
    for _ in range(3):
        s = s + (1.0 / 3.0) * D(s, Z, c, dt, dx, dy, cd)
    return (0.25 * q + 0.75 * s) + 0.25 * D(s, Z, c, dt, dx, dy, cd)


def rk(ti):
    return {1: ssp22, 2: ssp42, 3: ssprk3, 4: ssp104}[ti]
