"""CPU oracle of the projection steps around the pressure solve (test
infrastructure only: the CUDA kernels of nga2_b200/csrc/projection.cu are
checked against it; nothing in the product imports it).

A numpy restatement, term for term, of:

* the pgrid metrics: naive extension of the nodes over one overlap layer,
  cell sizes dx = x(i+1) - x(i), dxi = 1/dx, centroid spacings
  dxmi = 1/(xm(i) - xm(i-1))  (src/grid/sgrid_class.f90:160-254);
* divp_x = dxi*[-1, +1] on cells and divu_x = dxmi*[-1, +1] on faces
  (src/constant_density/incomp_class.f90:355-380), divu = 0 on the wall faces
  of non-periodic directions (umask = 2, incomp_class.f90:529-563);
* update_laplacian (src/two_phase/tpns_class.f90:1565-1593);
* get_div (incomp_class.f90:1144-1159) and rhs = -vol*div*rho/dt
  (examples/channel/src/simulation.f90:318);
* shift_p (incomp_class.f90:1720-1740) with cfg%integrate
  (src/config/config_class.f90:196-214, a sequential loop) and
  fluid_vol = xL*yL*zL (sgrid_class.f90:260-263);
* get_pgrad (incomp_class.f90:1163-1184);
* the velocity correction of examples/falling_drop/src/simulation.f90:308-313;
* cfg%sync on one rank: periodic images in the overlap.

Arrays are padded numpy arrays [k, j, i] with ``g`` overlap layers; the
operator is [k, j, i, 7].
"""
from __future__ import annotations

import numpy as np


def axis_metrics(x, per):
    """(divp(0), divp(1)) on the n cells, (divu(-1), divu(0)) on the n+1 faces
    and the cell sizes, for node coordinates x[0..n]."""
    x = np.asarray(x, np.float64)
    n = x.size - 1
    xe = np.empty(n + 3)
    xe[1:n + 2] = x
    xe[0] = xe[1] - (xe[2] - xe[1])
    xe[n + 2] = xe[n + 1] + (xe[n + 1] - xe[n])
    xm = 0.5 * (xe[:-1] + xe[1:])
    d = xe[2:n + 2] - xe[1:n + 1]
    di = 1.0 / d
    dmi = 1.0 / (xm[1:] - xm[:-1])
    du0, du1 = dmi * -1.0, dmi * 1.0
    if not per:
        du0[0] = du0[-1] = 0.0
        du1[0] = du1[-1] = 0.0
    return di * -1.0, di * 1.0, du0, du1, d


class Grid:
    def __init__(self, xn, yn, zn, per, g=1):
        self.xn, self.yn, self.zn = (np.asarray(a, np.float64) for a in (xn, yn, zn))
        self.nx, self.ny, self.nz = self.xn.size - 1, self.yn.size - 1, self.zn.size - 1
        self.per = tuple(bool(p) for p in per)
        self.g = g
        self.mx = axis_metrics(self.xn, self.per[0])
        self.my = axis_metrics(self.yn, self.per[1])
        self.mz = axis_metrics(self.zn, self.per[2])
        dx, dy, dz = self.mx[4], self.my[4], self.mz[4]
        self.vol = (dx[None, None, :] * dy[None, :, None]) * dz[:, None, None]
        self.vol_total = ((self.xn[-1] - self.xn[0]) * (self.yn[-1] - self.yn[0])) * (self.zn[-1] - self.zn[0])

    @property
    def padded(self):
        g = self.g
        return (self.nz + 2 * g, self.ny + 2 * g, self.nx + 2 * g)

    def interior(self, a, di=0, dj=0, dk=0):
        """View of the padded array shifted by (di, dj, dk) over the interior."""
        g = self.g
        return a[g + dk:g + dk + self.nz, g + dj:g + dj + self.ny, g + di:g + di + self.nx]

    def sync(self, a):
        """cfg%sync on one rank: x, then y, then z, each over the full extent."""
        g = self.g
        a = a.copy()
        if self.per[0]:
            n = self.nx
            a[:, :, :g] = a[:, :, n:n + g]
            a[:, :, n + g:] = a[:, :, g:2 * g]
        if self.per[1]:
            n = self.ny
            a[:, :g, :] = a[:, n:n + g, :]
            a[:, n + g:, :] = a[:, g:2 * g, :]
        if self.per[2]:
            n = self.nz
            a[:g, :, :] = a[n:n + g, :, :]
            a[n + g:, :, :] = a[g:2 * g, :, :]
        return a


def laplacian(G, rho_U=None, rho_V=None, rho_W=None):
    """update_laplacian: opr[k, j, i, 0:7] on the interior (zero elsewhere)."""
    dp0x, dp1x, du0x, du1x, _ = G.mx
    dp0y, dp1y, du0y, du1y, _ = G.my
    dp0z, dp1z, du0z, du1z, _ = G.mz
    one = np.ones(G.padded)
    rU = one if rho_U is None else rho_U
    rV = one if rho_V is None else rho_V
    rW = one if rho_W is None else rho_W
    X = lambda a: a[None, None, :]
    Y = lambda a: a[None, :, None]
    Z = lambda a: a[:, None, None]
    rUp, rUm = G.interior(rU, di=1), G.interior(rU)
    rVp, rVm = G.interior(rV, dj=1), G.interior(rV)
    rWp, rWm = G.interior(rW, dk=1), G.interior(rW)
    t = [X(dp1x) * X(du0x[1:]) / rUp, X(dp0x) * X(du1x[:-1]) / rUm,
         Y(dp1y) * Y(du0y[1:]) / rVp, Y(dp0y) * Y(du1y[:-1]) / rVm,
         Z(dp1z) * Z(du0z[1:]) / rWp, Z(dp0z) * Z(du1z[:-1]) / rWm]
    o = np.zeros(G.padded + (7,))
    g = G.g
    core = o[g:g + G.nz, g:g + G.ny, g:g + G.nx]
    core[..., 0] = ((((t[0] + t[1]) + t[2]) + t[3]) + t[4]) + t[5]
    core[..., 1] = X(dp1x) * X(du1x[1:]) / rUp
    core[..., 2] = X(dp0x) * X(du0x[:-1]) / rUm
    core[..., 3] = Y(dp1y) * Y(du1y[1:]) / rVp
    core[..., 4] = Y(dp0y) * Y(du0y[:-1]) / rVm
    core[..., 5] = Z(dp1z) * Z(du1z[1:]) / rWp
    core[..., 6] = Z(dp0z) * Z(du0z[:-1]) / rWm
    core[...] = -core * G.vol[..., None]
    return o


def divergence(G, U, V, W, rho=1.0, dt=None, div_out=None, rhs_out=None):
    """get_div (synchronised) and rhs = -vol*div*rho/dt on the interior."""
    dp0x, dp1x = G.mx[0], G.mx[1]
    dp0y, dp1y = G.my[0], G.my[1]
    dp0z, dp1z = G.mz[0], G.mz[1]
    sx = dp0x[None, None, :] * G.interior(U) + dp1x[None, None, :] * G.interior(U, di=1)
    sy = dp0y[None, :, None] * G.interior(V) + dp1y[None, :, None] * G.interior(V, dj=1)
    sz = dp0z[:, None, None] * G.interior(W) + dp1z[:, None, None] * G.interior(W, dk=1)
    d = (sx + sy) + sz
    div = np.zeros(G.padded) if div_out is None else div_out.copy()
    G.interior(div)[...] = d
    div = G.sync(div)
    rhs = None
    if dt is not None:
        rhs = np.zeros(G.padded) if rhs_out is None else rhs_out.copy()
        G.interior(rhs)[...] = -(((G.vol * d) * rho) / dt)
    return div, rhs


def shift_p(G, p):
    """(shifted and synchronised pressure, mean): the volume integral is the
    reference's sequential sum in loop order (i fastest)."""
    vals = (G.vol * 1.0) * G.interior(p)
    integral = np.cumsum(vals.reshape(-1))[-1]
    mean = integral / G.vol_total
    q = p.copy()
    G.interior(q)[...] = G.interior(p) - mean
    return G.sync(q), mean


def pgrad(G, P):
    du0x, du1x = G.mx[2], G.mx[3]
    du0y, du1y = G.my[2], G.my[3]
    du0z, du1z = G.mz[2], G.mz[3]
    gx, gy, gz = np.zeros(G.padded), np.zeros(G.padded), np.zeros(G.padded)
    G.interior(gx)[...] = du0x[None, None, :-1] * G.interior(P, di=-1) + du1x[None, None, :-1] * G.interior(P)
    G.interior(gy)[...] = du0y[None, :-1, None] * G.interior(P, dj=-1) + du1y[None, :-1, None] * G.interior(P)
    G.interior(gz)[...] = du0z[:-1, None, None] * G.interior(P, dk=-1) + du1z[:-1, None, None] * G.interior(P)
    return G.sync(gx), G.sync(gy), G.sync(gz)


def correct(G, sol, dt, U, V, W, P=None, rho_U=None, rho_V=None, rho_W=None):
    """P += sol; U -= dt*gradx/rho_U; ... on the interior, then synchronised."""
    gx, gy, gz = pgrad(G, sol)
    out = []
    for a, gr, r in ((U, gx, rho_U), (V, gy, rho_V), (W, gz, rho_W)):
        b = a.copy()
        rr = 1.0 if r is None else G.interior(r)
        G.interior(b)[...] = G.interior(a) - (dt * G.interior(gr)) / rr
        out.append(G.sync(b))
    if P is not None:
        q = P.copy()
        G.interior(q)[...] = G.interior(P) + G.interior(sol)
        out.append(G.sync(q))
    return out
