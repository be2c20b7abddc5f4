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
* get_dmomdt (incomp_class.f90:1021-1159) on triply periodic grids, with the
  metrics extended over two layers;
* the whole-array updates of a sub-iteration of examples/hit/src/simulation.f90
  (mid-time velocity, explicit residual with the linear forcing) and the flow
  statistics the loop needs (get_cfl, the kinetic energy, mean velocities);
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


# ----------------------------------------------------------------------------- momentum
def momentum_metrics(x):
    """Extended 1-D metrics of one periodic direction for get_dmomdt: cell
    sizes' inverses dxi on cells -1..n (index c+1), centroid spacings' inverses
    dxmi and the edge interpolation weights itp(-1), itp(0) on faces 0..n
    (incomp_class.f90:250-446, sgrid_class.f90:160-254 with two layers of the
    naive extension)."""
    x = np.asarray(x, np.float64)
    n = x.size - 1
    xe = np.empty(n + 5)              # nodes -2 .. n+2 at index +2
    xe[2:n + 3] = x
    for m in (1, 0):                  # x(i) = x(i+1) - (x(imin+1) - x(imin))
        xe[m] = xe[m + 1] - (xe[3] - xe[2])
    for m in (n + 3, n + 4):          # x(i) = x(i-1) + (x(imax+1) - x(imax))
        xe[m] = xe[m - 1] + (xe[n + 2] - xe[n + 1])
    xm = 0.5 * (xe[:-1] + xe[1:])     # cells -2 .. n+1 at index +2
    dx = xe[1:] - xe[:-1]
    dxi = (1.0 / dx)[1:n + 3]         # cells -1 .. n
    f = np.arange(0, n + 1)           # faces 0 .. n
    dxmi = 1.0 / (xm[f + 2] - xm[f + 1])
    itm = dxmi * (xm[f + 2] - xe[f + 2])   # weight of the value at index f-1
    itz = dxmi * (xe[f + 2] - xm[f + 1])   # weight of the value at index f
    return dxi, dxmi, itm, itz


def dmomdt(G, U, V, W, P, rho, visc):
    """get_dmomdt (incomp_class.f90:1021-1159) on a triply periodic grid: the
    time derivatives of rho U, rho V, rho W on the interior faces, term for
    term (constant density rho, cell-centred viscosity array visc).  Ghost
    layers of U, V, W, P and visc must hold the periodic images."""
    assert all(G.per), "periodic directions only"
    mx, my, mz = (momentum_metrics(a) for a in (G.xn, G.yn, G.zn))
    nx, ny, nz = G.nx, G.ny, G.nz
    c23 = 2.0 / 3.0

    def A(a, dx=0, dy=0, dz=0):
        return G.interior(a, di=dx, dj=dy, dk=dz)

    def cx(m, off):   # cell metric at interior index + off, broadcast along x
        return m[0][1 + off:1 + off + nx][None, None, :]

    def cy(m, off):
        return m[0][1 + off:1 + off + ny][None, :, None]

    def cz(m, off):
        return m[0][1 + off:1 + off + nz][:, None, None]

    def fx(m, q, off):  # face metric q (1 dxmi, 2 itm, 3 itz) at face i + off
        return m[q][off:off + nx][None, None, :]

    def fy(m, q, off):
        return m[q][off:off + ny][None, :, None]

    def fz(m, q, off):
        return m[q][off:off + nz][:, None, None]

    def two(a0, b0, a1, b1):  # sum(a(:)*b(:)) of two terms
        return a0 * b0 + a1 * b1

    # divergence at a cell, the divp sums of the normal fluxes
    def divc(ox, oy, oz):
        dxi, dyi, dzi = cx(mx, ox), cy(my, oy), cz(mz, oz)
        sx = two(dxi * -1.0, A(U, ox, oy, oz), dxi * 1.0, A(U, ox + 1, oy, oz))
        sy = two(dyi * -1.0, A(V, ox, oy, oz), dyi * 1.0, A(V, ox, oy + 1, oz))
        sz = two(dzi * -1.0, A(W, ox, oy, oz), dzi * 1.0, A(W, ox, oy, oz + 1))
        return (sx + sy) + sz

    def normal(Q, d, off):  # FX of rhoU (d=0), FY of rhoV (1), FZ of rhoW (2) at cell + off along d
        o = [0, 0, 0]
        o[d] = off
        m = (mx, my, mz)[d]
        ci = (cx, cy, cz)[d](m, off)
        sh = [0, 0, 0]
        sh[d] = 1
        q0, q1 = A(Q, *o), A(Q, o[0] + sh[0], o[1] + sh[1], o[2] + sh[2])
        s1 = two(0.5, q0, 0.5, q1)
        g = two(ci * -1.0, q0, ci * 1.0, q1)
        return ((-(rho * s1 * s1)) + A(visc, *o) * ((g + g) - c23 * divc(*o))) - A(P, *o)

    def edge(d1, d2, o1, o2, Qa, Qb):
        """Edge flux in the (d1, d2) plane at face offsets o1 (along d1), o2 (along d2):
        -rho (itp_{d1} Qa) (itp_{d2} Qb) + (itp_2d visc) (grd_{d1} Qa + grd_{d2} Qb), where Qa
        varies along d1 and Qb along d2; the 2-D viscosity sum runs over (s1 along d1,
        s2 along d2) in Fortran order (first index fastest) of the reference's itp_xy/yz/xz."""
        o = [0, 0, 0]
        o[d1] += o1
        o[d2] += o2
        m1, m2 = (mx, my, mz)[d1], (mx, my, mz)[d2]
        f1, f2 = (fx, fy, fz)[d1], (fx, fy, fz)[d2]
        e1 = [0, 0, 0]
        e1[d1] = -1
        e2 = [0, 0, 0]
        e2[d2] = -1
        qa_m = A(Qa, o[0] + e1[0], o[1] + e1[1], o[2] + e1[2])
        qa_0 = A(Qa, *o)
        qb_m = A(Qb, o[0] + e2[0], o[1] + e2[1], o[2] + e2[2])
        qb_0 = A(Qb, *o)
        a = two(f1(m1, 2, o1), qa_m, f1(m1, 3, o1), qa_0)
        b = two(f2(m2, 2, o2), qb_m, f2(m2, 3, o2), qb_0)
        return a, b, qa_m, qa_0, qb_m, qb_0, o, (m1, f1, o1), (m2, f2, o2)

    def visc2(dlo, dhi, o, wlo, whi):
        # itp_2d(st_lo, st_hi) = itp_lo(st_lo) itp_hi(st_hi) (incomp_class.f90:277-288), rescaled
        # by its sum in adjust_metrics (incomp_class.f90:505-511); then sum(itp_2d * visc(..)),
        # both sums over (st_lo, st_hi) in {-1,0}^2 with st_lo fastest
        (mlo, flo, olo), (mhi, fhi, ohi) = wlo, whi
        itl = {-1: flo(mlo, 2, olo), 0: flo(mlo, 3, olo)}
        ith = {-1: fhi(mhi, 2, ohi), 0: fhi(mhi, 3, ohi)}
        order = [(sl, sh) for sh in (-1, 0) for sl in (-1, 0)]
        w = {key: itl[key[0]] * ith[key[1]] for key in order}
        mysum = ((w[order[0]] + w[order[1]]) + w[order[2]]) + w[order[3]]
        assert np.all(mysum > 0.0)
        w = {key: val / mysum for key, val in w.items()}
        s = None
        for sl, sh in order:
            p = list(o)
            p[dlo] += sl
            p[dhi] += sh
            t = w[(sl, sh)] * A(visc, *p)
            s = t if s is None else s + t
        return s

    def grd(m, f, off, q_m, q_0):
        dmi = f(m, 1, off)
        return two(dmi * -1.0, q_m, dmi * 1.0, q_0)

    # ---- rho U: FX at cells i-1, i; FY at xy edges (i, j), (i, j+1); FZ at xz edges (i, k), (i, k+1)
    FX = [normal(U, 0, -1), normal(U, 0, 0)]
    FY, FZ = [], []
    for oy in (0, 1):
        a, b, qa_m, qa_0, qb_m, qb_0, o, w1, w2 = edge(1, 0, oy, 0, U, V)   # a: itpu_y U, b: itpv_x V
        vi = visc2(0, 1, o, w2, w1)                                           # itp_xy(x fastest, y)
        g = grd(*w1[:2], w1[2], qa_m, qa_0) + grd(*w2[:2], w2[2], qb_m, qb_0)
        FY.append((-(rho * a * b)) + vi * g)
    for oz in (0, 1):
        a, b, qa_m, qa_0, qb_m, qb_0, o, w1, w2 = edge(2, 0, oz, 0, U, W)   # a: itpu_z U, b: itpw_x W
        vi = visc2(0, 2, o, w2, w1)                                           # itp_xz(x fastest, z)
        g = grd(*w1[:2], w1[2], qa_m, qa_0) + grd(*w2[:2], w2[2], qb_m, qb_0)
        FZ.append((-(rho * a * b)) + vi * g)
    dmx = fx(mx, 1, 0)
    dU = (two(dmx * -1.0, FX[0], dmx * 1.0, FX[1]) + two(cy(my, 0) * -1.0, FY[0], cy(my, 0) * 1.0, FY[1])) \
        + two(cz(mz, 0) * -1.0, FZ[0], cz(mz, 0) * 1.0, FZ[1])

    # ---- rho V: FX at xy edges (i, j), (i+1, j); FY at cells j-1, j; FZ at yz edges (j, k), (j, k+1)
    FX, FZ = [], []
    for ox in (0, 1):
        a, b, qa_m, qa_0, qb_m, qb_0, o, w1, w2 = edge(0, 1, ox, 0, V, U)   # a: itpv_x V, b: itpu_y U
        vi = visc2(0, 1, o, w1, w2)
        g = grd(*w1[:2], w1[2], qa_m, qa_0) + grd(*w2[:2], w2[2], qb_m, qb_0)
        FX.append((-(rho * a * b)) + vi * g)
    FY = [normal(V, 1, -1), normal(V, 1, 0)]
    for oz in (0, 1):
        a, b, qa_m, qa_0, qb_m, qb_0, o, w1, w2 = edge(2, 1, oz, 0, V, W)   # a: itpv_z V, b: itpw_y W
        vi = visc2(1, 2, o, w2, w1)                                           # itp_yz(y fastest, z)
        g = grd(*w1[:2], w1[2], qa_m, qa_0) + grd(*w2[:2], w2[2], qb_m, qb_0)
        FZ.append((-(rho * a * b)) + vi * g)
    dmy = fy(my, 1, 0)
    dV = (two(cx(mx, 0) * -1.0, FX[0], cx(mx, 0) * 1.0, FX[1]) + two(dmy * -1.0, FY[0], dmy * 1.0, FY[1])) \
        + two(cz(mz, 0) * -1.0, FZ[0], cz(mz, 0) * 1.0, FZ[1])

    # ---- rho W: FX at xz edges (i, k), (i+1, k); FY at yz edges (j, k), (j+1, k); FZ at cells k-1, k
    FX, FY = [], []
    for ox in (0, 1):
        a, b, qa_m, qa_0, qb_m, qb_0, o, w1, w2 = edge(0, 2, ox, 0, W, U)   # a: itpw_x W, b: itpu_z U
        vi = visc2(0, 2, o, w1, w2)
        g = grd(*w1[:2], w1[2], qa_m, qa_0) + grd(*w2[:2], w2[2], qb_m, qb_0)
        FX.append((-(rho * a * b)) + vi * g)
    for oy in (0, 1):
        a, b, qa_m, qa_0, qb_m, qb_0, o, w1, w2 = edge(1, 2, oy, 0, W, V)   # a: itpw_y W, b: itpv_z V
        vi = visc2(1, 2, o, w1, w2)
        g = grd(*w1[:2], w1[2], qa_m, qa_0) + grd(*w2[:2], w2[2], qb_m, qb_0)
        FY.append((-(rho * a * b)) + vi * g)
    FZ = [normal(W, 2, -1), normal(W, 2, 0)]
    dmz = fz(mz, 1, 0)
    dW = (two(cx(mx, 0) * -1.0, FX[0], cx(mx, 0) * 1.0, FX[1]) + two(cy(my, 0) * -1.0, FY[0], cy(my, 0) * 1.0, FY[1])) \
        + two(dmz * -1.0, FZ[0], dmz * 1.0, FZ[1])
    out = []
    for d in (dU, dV, dW):
        a = np.zeros(G.padded)
        G.interior(a)[...] = d
        out.append(G.sync(a))
    return out


def midpoint(U, Uold):
    """fs%U=0.5_WP*(fs%U+fs%Uold) (examples/hit/src/simulation.f90:283-285),
    whole padded arrays."""
    return 0.5 * (U + Uold)


def advance(dt, rho, U, Uold, dU, force_a=0.0, force_b=1.0, mean=0.0):
    """The explicit update of a sub-iteration (examples/hit/src/simulation.f90:
    291-325) for one component over the whole padded array: resU =
    -2*(rho*U - rho*Uold) + dt*resU, plus the linear forcing
    (force_a*(U - mean))/force_b when force_a != 0, then U = 2*U - Uold + resU/rho."""
    res = -2.0 * (rho * U - rho * Uold) + dt * dU
    if force_a != 0.0:
        res = res + (force_a * (U - mean)) / force_b
    return (2.0 * U - Uold) + res / rho


def flow_stats(G, U, V, W, visc, rho, dt):
    """get_cfl's six CFLs (incomp_class.f90:1497-1540), the kinetic energy of
    interp_vel's cell velocities (incomp_class.f90:1188-1225, summed as in
    examples/hit/src/simulation.f90:299-311) and the volume means of U, V, W
    (config_class.f90:196-214 over fluid_vol), triply periodic grids."""
    mx, my, mz = (momentum_metrics(a) for a in (G.xn, G.yn, G.zn))
    nx, ny, nz = G.nx, G.ny, G.nz
    u, v, w, vis = G.interior(U), G.interior(V), G.interior(W), G.interior(visc)
    cflc = [(np.abs(u) * mx[1][:nx][None, None, :]).max() * dt,
            (np.abs(v) * my[1][:ny][None, :, None]).max() * dt,
            (np.abs(w) * mz[1][:nz][:, None, None]).max() * dt]
    dxi, dyi, dzi = mx[0][1:nx + 1], my[0][1:ny + 1], mz[0][1:nz + 1]
    cflv = [((4.0 * vis) * (dxi * dxi)[None, None, :] / rho).max() * dt,
            ((4.0 * vis) * (dyi * dyi)[None, :, None] / rho).max() * dt,
            ((4.0 * vis) * (dzi * dzi)[:, None, None] / rho).max() * dt]
    ui = 0.5 * u + 0.5 * G.interior(U, di=1)
    vi = 0.5 * v + 0.5 * G.interior(V, dj=1)
    wi = 0.5 * w + 0.5 * G.interior(W, dk=1)
    ke = (0.5 * ((ui * ui + vi * vi) + wi * wi)).sum()
    vol = G.vol
    means = [(vol * a).sum() / G.vol_total for a in (u, v, w)]
    return np.array(cflc + cflv + [ke] + means)


class HITOracle:
    """examples/hit/src/simulation.f90 on the CPU (lines 100-135 for the
    initial field, 256-352 for the time loop; no particles), built from the
    functions above and a pressure solve ``solve(opr, rhs) -> sol`` on
    interior arrays (the oracle bbmg in the tests).  dt follows
    timetracker_class.f90:88-97 (adjust_dt, alpha = 0.7) and 68-84."""

    def __init__(self, n, solve, Lx=1.0, visc=0.01, rho=1.0, urms0=5.0, tau_eddy=0.1, dtmax=1e-3, cflmax=0.9,
                 itmax=2, seed=0, g=1, forcing=True):
        x = np.arange(n + 1, dtype=np.float64) / float(n) * Lx
        self.G = G = Grid(x, x, x, (True, True, True), g)
        self.solve, self.rho, self.tau, self.forcing = solve, float(rho), float(tau_eddy), forcing
        self.visc = np.full(G.padded, float(visc))
        self.rho_face = np.full(G.padded, self.rho)
        self.opr = laplacian(G)
        self.dtmax, self.cflmax, self.itmax = dtmax, cflmax, itmax
        self.dt, self.t, self.n, self.cfl = dtmax, 0.0, 0, 0.0
        rng = np.random.default_rng(seed)
        self.U, self.V, self.W = (self._fill(rng.normal(0.0, urms0, size=(n, n, n))) for _ in range(3))
        self.P = np.zeros(G.padded)
        self.sol = np.zeros(G.padded)
        self._project(self.dt)
        self.KE0 = flow_stats(G, self.U, self.V, self.W, self.visc, self.rho, 1.0)[6]

    def _fill(self, inner):
        a = np.zeros(self.G.padded)
        self.G.interior(a)[...] = inner
        return self.G.sync(a)

    def _project(self, dt):
        G = self.G
        _, rhs = divergence(G, self.U, self.V, self.W, rho=self.rho, dt=dt)
        x = self.solve(np.ascontiguousarray(G.interior(self.opr)), np.ascontiguousarray(G.interior(rhs)))
        sol = self._fill(x)
        sol, _ = shift_p(G, sol)
        self.sol = sol
        self.U, self.V, self.W, self.P = correct(G, sol, dt, self.U, self.V, self.W, self.P, self.rho_face,
                                                 self.rho_face, self.rho_face)

    def step(self):
        G = self.G
        s = flow_stats(G, self.U, self.V, self.W, self.visc, self.rho, self.dt)
        self.cfl = s[:6].max()
        dtold = self.dt
        if self.cfl > 0.0:
            self.dt = min(dtold * self.cflmax / self.cfl, self.dtmax)
        if self.dt > dtold:
            self.dt = 0.7 * self.dt + (1.0 - 0.7) * dtold
        self.t += self.dt
        self.n += 1
        dt = self.dt
        Uo, Vo, Wo = self.U.copy(), self.V.copy(), self.W.copy()
        for _ in range(self.itmax):
            self.U, self.V, self.W = midpoint(self.U, Uo), midpoint(self.V, Vo), midpoint(self.W, Wo)
            dU, dV, dW = dmomdt(G, self.U, self.V, self.W, self.P, self.rho, self.visc)
            fa, mean = 0.0, (0.0, 0.0, 0.0)
            if self.forcing:
                st = flow_stats(G, self.U, self.V, self.W, self.visc, self.rho, 1.0)
                fa, mean = dt * self.KE0 / st[6], st[7:10]
            self.U = advance(dt, self.rho, self.U, Uo, dU, fa, 2.0 * self.tau, mean[0])
            self.V = advance(dt, self.rho, self.V, Vo, dV, fa, 2.0 * self.tau, mean[1])
            self.W = advance(dt, self.rho, self.W, Wo, dW, fa, 2.0 * self.tau, mean[2])
            self._project(dt)
