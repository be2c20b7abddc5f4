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
def momentum_metrics(x, walls=False):
    """Extended 1-D metrics of one direction for get_dmomdt: cell sizes'
    inverses dxi on cells -1..n (index c+1); on faces 0..n the centroid
    spacings' inverses dxmi and the edge interpolation weights itm, itz (of
    the values at f-1 and f) (incomp_class.f90:250-446, sgrid_class.f90:
    160-254 with two layers of the naive extension); then the adjust_metrics
    versions (incomp_class.f90:449-700) for walls at both ends of a
    non-periodic direction (cfg%VF = 0 outside the domain): vtm, vtz, gdm,
    the interpolation weights and gradient coefficient of a velocity
    component tangential to the direction ([1,0], [0,1] and 1/delta on the
    wall faces), and wtm, wtz, the 1-D factors of the edge viscosity weights
    with the wall cell's entry zeroed."""
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
    vtm, vtz, gdm, wtm, wtz = itm.copy(), itz.copy(), dxmi.copy(), itm.copy(), itz.copy()
    if walls:
        vtm[0], vtz[0], gdm[0] = 1.0, 0.0, 1.0 / (xm[2] - xe[2])              # delta = xm(0) - x(0)
        vtm[n], vtz[n], gdm[n] = 0.0, 1.0, 1.0 / (xe[n + 2] - xm[n + 1])      # delta = x(n) - xm(n-1)
        wtm[0] = 0.0                                                          # cell -1 is wall
        wtz[n] = 0.0                                                          # cell n is wall
    dm = xm[f + 2] - xm[f + 1]        # cfg%dxm on faces 0 .. n
    return dxi, dxmi, itm, itz, vtm, vtz, gdm, wtm, wtz, dm


def dmomdt(G, U, V, W, P, rho, visc):
    """get_dmomdt (incomp_class.f90:1021-1159): the time derivatives of rho U,
    rho V, rho W on the interior faces, term for term (constant density rho,
    cell-centred viscosity array visc).  A non-periodic direction has walls
    at both ends (cfg%VF = 0 outside the domain): edge coefficients from
    adjust_metrics and a zero derivative of the wall-normal component on the
    wall faces (divu = 0 where umask > 0).  Ghost layers of periodic
    directions must hold the periodic images."""
    walls = [not p for p in G.per]
    ms = [momentum_metrics(a, w) for a, w in zip((G.xn, G.yn, G.zn), walls)]
    nx, ny, nz = G.nx, G.ny, G.nz
    ns = (nx, ny, nz)
    c23 = 2.0 / 3.0

    def A(a, dx=0, dy=0, dz=0):
        return G.interior(a, di=dx, dj=dy, dk=dz)

    def shape(d, v):  # broadcast a 1-D array along direction d
        return v[None, None, :] if d == 0 else (v[None, :, None] if d == 1 else v[:, None, None])

    def cell(d, off):  # dxi of direction d at interior cell index + off
        return shape(d, ms[d][0][1 + off:1 + off + ns[d]])

    def face(d, q, off):  # face metric q of direction d at interior index + off
        return shape(d, ms[d][q][off:off + ns[d]])

    def wall_face(d, off):  # the face (interior index + off) along d lies on a wall
        idx = np.arange(off, off + ns[d])
        return shape(d, walls[d] & ((idx == 0) | (idx == ns[d])))

    def two(a0, b0, a1, b1):  # sum(a(:)*b(:)) of two terms
        return a0 * b0 + a1 * b1

    def shifted(o, d, s):
        p = list(o)
        p[d] += s
        return p

    # divergence at a cell, the divp sums of the normal fluxes
    def divc(ox, oy, oz):
        dxi, dyi, dzi = cell(0, ox), cell(1, oy), cell(2, oz)
        sx = two(dxi * -1.0, A(U, ox, oy, oz), dxi * 1.0, A(U, ox + 1, oy, oz))
        sy = two(dyi * -1.0, A(V, ox, oy, oz), dyi * 1.0, A(V, ox, oy + 1, oz))
        sz = two(dzi * -1.0, A(W, ox, oy, oz), dzi * 1.0, A(W, ox, oy, oz + 1))
        return (sx + sy) + sz

    def normal(Q, d, off):  # FX of rhoU (d=0), FY of rhoV (1), FZ of rhoW (2) at cell + off along d
        o = shifted([0, 0, 0], d, off)
        ci = cell(d, off)
        q0, q1 = A(Q, *o), A(Q, *shifted(o, d, 1))
        s1 = two(0.5, q0, 0.5, q1)
        g = two(ci * -1.0, q0, ci * 1.0, q1)
        return ((-(rho * s1 * s1)) + A(visc, *o) * ((g + g) - c23 * divc(*o))) - A(P, *o)

    def tang(d, off, cw):
        """Interpolation weights and gradient pair along d at face + off of a
        component whose own face is a wall face (cw) or not."""
        tm = np.where(cw, face(d, 2, off), face(d, 4, off))
        tz = np.where(cw, face(d, 3, off), face(d, 5, off))
        g = face(d, 6, off)
        return tm, tz, np.where(cw, 0.0, -g), np.where(cw, 0.0, g)

    def edge(d1, o1, d2, o2, Qa, Qb):
        """Edge flux in the (d1, d2) plane at face offsets o1 (along d1), o2 (along d2),
        Qa the component along d2 varying along d1, Qb the component along d1 varying
        along d2: -rho (itp_d1 Qa) (itp_d2 Qb) + (itp_2d visc) (grd_d1 Qa + grd_d2 Qb)."""
        o = shifted(shifted([0, 0, 0], d1, o1), d2, o2)
        qa_m, qa_0 = A(Qa, *shifted(o, d1, -1)), A(Qa, *o)
        qb_m, qb_0 = A(Qb, *shifted(o, d2, -1)), A(Qb, *o)
        am, az, gam, gaz = tang(d1, o1, wall_face(d2, o2))
        bm, bz, gbm, gbz = tang(d2, o2, wall_face(d1, o1))
        a = two(am, qa_m, az, qa_0)
        b = two(bm, qb_m, bz, qb_0)
        g = two(gam, qa_m, gaz, qa_0) + two(gbm, qb_m, gbz, qb_0)
        # itp_2d(st_lo, st_hi) = itp_lo(st_lo) itp_hi(st_hi) (incomp_class.f90:277-288), wall
        # cells' entries zeroed and the rest rescaled by the sum (adjust_metrics,
        # incomp_class.f90:497-511); sums over (st_lo, st_hi) with st_lo fastest
        (dlo, olo), (dhi, ohi) = sorted(((d1, o1), (d2, o2)))
        itl = {-1: face(dlo, 7, olo), 0: face(dlo, 8, olo)}
        ith = {-1: face(dhi, 7, ohi), 0: face(dhi, 8, ohi)}
        order = [(sl, sh) for sh in (-1, 0) for sl in (-1, 0)]
        w = {key: itl[key[0]] * ith[key[1]] for key in order}
        mysum = ((w[order[0]] + w[order[1]]) + w[order[2]]) + w[order[3]]
        assert np.all(mysum > 0.0)
        vi = None
        for sl, sh in order:
            t = (w[(sl, sh)] / mysum) * A(visc, *shifted(shifted(o, dlo, sl), dhi, sh))
            vi = t if vi is None else vi + t
        return (-(rho * a * b)) + vi * g

    # ---- rho U: FX at cells i-1, i; FY at xy edges (i, j), (i, j+1); FZ at xz edges (i, k), (i, k+1)
    FX = [normal(U, 0, -1), normal(U, 0, 0)]
    FY = [edge(1, oy, 0, 0, U, V) for oy in (0, 1)]
    FZ = [edge(2, oz, 0, 0, U, W) for oz in (0, 1)]
    dmx, dy, dz = face(0, 1, 0), cell(1, 0), cell(2, 0)
    dU = (two(dmx * -1.0, FX[0], dmx * 1.0, FX[1]) + two(dy * -1.0, FY[0], dy * 1.0, FY[1])) \
        + two(dz * -1.0, FZ[0], dz * 1.0, FZ[1])
    dU = np.where(wall_face(0, 0), 0.0, dU)

    # ---- rho V: FX at xy edges (i, j), (i+1, j); FY at cells j-1, j; FZ at yz edges (j, k), (j, k+1)
    FX = [edge(0, ox, 1, 0, V, U) for ox in (0, 1)]
    FY = [normal(V, 1, -1), normal(V, 1, 0)]
    FZ = [edge(2, oz, 1, 0, V, W) for oz in (0, 1)]
    dx, dmy = cell(0, 0), face(1, 1, 0)
    dV = (two(dx * -1.0, FX[0], dx * 1.0, FX[1]) + two(dmy * -1.0, FY[0], dmy * 1.0, FY[1])) \
        + two(dz * -1.0, FZ[0], dz * 1.0, FZ[1])
    dV = np.where(wall_face(1, 0), 0.0, dV)

    # ---- rho W: FX at xz edges (i, k), (i+1, k); FY at yz edges (j, k), (j+1, k); FZ at cells k-1, k
    FX = [edge(0, ox, 2, 0, W, U) for ox in (0, 1)]
    FY = [edge(1, oy, 2, 0, W, V) for oy in (0, 1)]
    FZ = [normal(W, 2, -1), normal(W, 2, 0)]
    dmz = face(2, 1, 0)
    dW = (two(dx * -1.0, FX[0], dx * 1.0, FX[1]) + two(dy * -1.0, FY[0], dy * 1.0, FY[1])) \
        + two(dmz * -1.0, FZ[0], dmz * 1.0, FZ[1])
    dW = np.where(wall_face(2, 0), 0.0, dW)
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


def implicit_operator(G, comp, dt, rho, U, V, W, visc):
    """The 7-point operator solve_implicit assembles for velocity component
    comp (0 U, 1 V, 2 W) (incomp_class.f90:1744-1910): rho on the diagonal
    plus 0.5*dt times the linearised convective terms, minus 0.5*dt times the
    viscous terms, in NGA2's stencil order [0, +x, -x, +y, -y, +z, -z]; the
    interior of a (nz, ny, nx, 7) array.  Walls as in dmomdt: the metrics of
    non-periodic directions carry adjust_metrics' wall coefficients and the
    rows of the component's wall faces are rho alone."""
    walls = [not p for p in G.per]
    ms = [momentum_metrics(a, w) for a, w in zip((G.xn, G.yn, G.zn), walls)]
    ns = (G.nx, G.ny, G.nz)
    Q = (U, V, W)
    c = comp

    def A(a, o):
        return G.interior(a, di=o[0], dj=o[1], dk=o[2])

    def shape(d, v):
        return v[None, None, :] if d == 0 else (v[None, :, None] if d == 1 else v[:, None, None])

    def cell(d, off):
        return shape(d, ms[d][0][1 + off:1 + off + ns[d]])

    def face(d, q, off):
        return shape(d, ms[d][q][off:off + ns[d]])

    def wall_face(d, off):
        idx = np.arange(off, off + ns[d])
        return shape(d, walls[d] & ((idx == 0) | (idx == ns[d])))

    def sh(d, s):
        o = [0, 0, 0]
        o[d] = s
        return o

    def add(o1, o2):
        return [a + b for a, b in zip(o1, o2)]

    def tang(d, off, cw):
        tm = np.where(cw, face(d, 2, off), face(d, 4, off))
        tz = np.where(cw, face(d, 3, off), face(d, 5, off))
        g = face(d, 6, off)
        return tm, tz, np.where(cw, 0.0, -g), np.where(cw, 0.0, g)

    def visc_edge(d, off):
        """Viscosity at the edge in the (c, d) plane at c-face 0 and d-face off."""
        (dlo, olo), (dhi, ohi) = sorted(((c, 0), (d, off)))
        itl = {-1: face(dlo, 7, olo), 0: face(dlo, 8, olo)}
        ith = {-1: face(dhi, 7, ohi), 0: face(dhi, 8, ohi)}
        order = [(sl, s2) for s2 in (-1, 0) for sl in (-1, 0)]
        w = {key: itl[key[0]] * ith[key[1]] for key in order}
        mysum = ((w[order[0]] + w[order[1]]) + w[order[2]]) + w[order[3]]
        base = sh(d, off)
        v = None
        for sl, s2 in order:
            t = (w[(sl, s2)] / mysum) * A(visc, add(add(base, sh(dlo, sl)), sh(dhi, s2)))
            v = t if v is None else v + t
        return v

    conv_d, conv_off = [], {}
    visc_d, visc_off = [], {}
    for d in range(3):
        if d == c:
            # normal: cells f (above) and f-1 (below) of the face; itpn = [0.5, 0.5] (0 in wall cells)
            def itpn(off):
                idx = np.arange(off, off + ns[c])
                wallcell = walls[c] & ((idx < 0) | (idx >= ns[c]))
                return shape(c, np.where(wallcell, 0.0, 0.5))
            rp = (rho * (itpn(0) * A(Q[c], [0, 0, 0]) + itpn(0) * A(Q[c], sh(c, 1)))) * 2.0
            rm = (rho * (itpn(-1) * A(Q[c], sh(c, -1)) + itpn(-1) * A(Q[c], [0, 0, 0]))) * 2.0
            dup, dlo = face(c, 1, 0), face(c, 1, 0) * -1.0
            tp, tm_ = (dup * itpn(0)) * rp, (dlo * itpn(-1)) * rm
            op, om = (dup * itpn(0)) * rp, (dlo * itpn(-1)) * rm
            ci0, cim = cell(c, 0), cell(c, -1)
            vp = (((dup * 4.0) / 3.0) * A(visc, [0, 0, 0])) * (ci0 * -1.0)
            vm = (((dlo * 4.0) / 3.0) * A(visc, sh(c, -1))) * (cim * 1.0)
            wp = (((dup * 4.0) / 3.0) * A(visc, [0, 0, 0])) * (ci0 * 1.0)
            wm = (((dlo * 4.0) / 3.0) * A(visc, sh(c, -1))) * (cim * -1.0)
        else:
            # tangential: edges at d-faces g+1 (upper) and g (lower) of the cell row
            cw_c = wall_face(c, 0)                       # the component's own face on a wall
            am_u, az_u, gm_u, gz_u = tang(d, 1, cw_c)    # Q_c along d at edge g+1
            am_l, az_l, gm_l, gz_l = tang(d, 0, cw_c)    # Q_c along d at edge g
            bm_u, bz_u, _, _ = tang(c, 0, wall_face(d, 1))  # Q_d along c at the c-face, edge g+1
            bm_l, bz_l, _, _ = tang(c, 0, wall_face(d, 0))
            qd = Q[d]
            rp = rho * (bm_u * A(qd, add(sh(c, -1), sh(d, 1))) + bz_u * A(qd, sh(d, 1)))
            rm = rho * (bm_l * A(qd, sh(c, -1)) + bz_l * A(qd, [0, 0, 0]))
            dup, dlo = cell(d, 0), cell(d, 0) * -1.0
            tp, tm_ = (dup * am_u) * rp, (dlo * az_l) * rm
            op, om = (dup * az_u) * rp, (dlo * am_l) * rm
            veu, vel = visc_edge(d, 1), visc_edge(d, 0)
            vp, vm = (dup * veu) * gm_u, (dlo * vel) * gz_l
            wp, wm = (dup * veu) * gz_u, (dlo * vel) * gm_l
        conv_d += [tp, tm_]
        visc_d += [vp, vm]
        conv_off[(d, 1)], conv_off[(d, -1)] = op, om
        visc_off[(d, 1)], visc_off[(d, -1)] = wp, wm
    hd = 0.5 * dt
    s = conv_d[0]
    for t in conv_d[1:]:
        s = s + t
    v = visc_d[0]
    for t in visc_d[1:]:
        v = v + t
    out = np.zeros((G.nz, G.ny, G.nx, 7))
    out[..., 0] = (rho + hd * s) - hd * v
    for q, key in enumerate([(0, 1), (0, -1), (1, 1), (1, -1), (2, 1), (2, -1)], start=1):
        out[..., q] = (0.0 + hd * conv_off[key]) - hd * visc_off[key]
    wf = wall_face(c, 0)
    out[..., 0] = np.where(wf, rho, out[..., 0])
    out[..., 1:] = np.where(wf[..., None], 0.0, out[..., 1:])
    return out


def extended_centres(x, g):
    """Cell centres xm of padded cells -g .. n+g-1 (the naive node extension)."""
    x = np.asarray(x, np.float64)
    n = x.size - 1
    xe = np.empty(n + 1 + 2 * g)
    xe[g:g + n + 1] = x
    for m in range(g - 1, -1, -1):
        xe[m] = xe[m + 1] - (xe[g + 1] - xe[g])
    for m in range(g + n + 1, n + 1 + 2 * g):
        xe[m] = xe[m - 1] + (xe[g + n] - xe[g + n - 1])
    return 0.5 * (xe[:-1] + xe[1:])


def face_mask(G, c):
    """umask (c = 0), vmask (1), wmask (2) > 0 on the padded array for walls
    at both ends of every non-periodic direction (incomp_class.f90:196-242
    with cfg%VF = 0 outside the domain)."""
    g, ns = G.g, (G.nx, G.ny, G.nz)
    m = np.zeros(G.padded, bool)
    for d in range(3):
        if G.per[d]:
            continue
        idx = np.arange(-g, ns[d] + g)
        md = ((idx <= 0) | (idx >= ns[d])) if d == c else ((idx < 0) | (idx >= ns[d]))
        m |= md[None, None, :] if d == 0 else (md[None, :, None] if d == 1 else md[:, None, None])
    return m


def mom_residual(G, c, dt, rho, U, Uold, res, force=None):
    """resU = -2*(rho*U - rho*Uold) + dt*resU, then (resU + a) - b where umask
    is 0 for force = (a, b) (examples/channel/src/simulation.f90:290-301)."""
    r = -2.0 * (rho * U - rho * Uold) + dt * res
    if force is not None:
        r = np.where(face_mask(G, c), r, (r + force[0]) - force[1])
    return r


def apply_residual(U, Uold, res):
    """U = 2*U - Uold + resU (examples/channel/src/simulation.f90:319-321)."""
    return (2.0 * U - Uold) + res


def bulk(G, c, U, Uold):
    """The channel forcing's sums (examples/channel/src/simulation.f90:
    280-298) for component c: sum over the interior faces with mask 0 of
    w*(2*U - Uold) and of w, w = dxm*dy*dz for U (dx*dym*dz, dx*dy*dzm)."""
    ns = (G.nx, G.ny, G.nz)
    w = None
    for d, xn in enumerate((G.xn, G.yn, G.zn)):
        v = momentum_metrics(xn, not G.per[d])[9][:ns[d]] if d == c else np.diff(np.asarray(xn, np.float64))
        v = v[None, None, :] if d == 0 else (v[None, :, None] if d == 1 else v[:, None, None])
        w = v if w is None else w * v
    w = np.broadcast_to(w, (G.nz, G.ny, G.nx))
    keep = ~G.interior(face_mask(G, c))
    return (w * (2.0 * G.interior(U) - G.interior(Uold)))[keep].sum(), w[keep].sum()


class ChannelOracle:
    """examples/channel/src/simulation.f90 on the CPU (initial field lines
    147-167, time loop 256-340) on its geometry (geometry.f90:30-61: x and z
    periodic, tanh-stretched y between walls), with solves
    ``solve_p(opr, rhs)`` (pressure) and ``solve_v(opr, rhs)`` (implicit
    velocity) on interior arrays."""

    def __init__(self, nx, ny, nz, solve_p, solve_v, Lx=5.0, Ly=1.0, Lz=0.04, stretch=2.1, visc=0.01, rho=1.0,
                 Ubulk=1.0, Wbulk=0.0, amp=0.0, dtmax=2e-2, cflmax=0.9, itmax=2, g=1, forcing=True):
        self.forcing = forcing
        x = np.arange(nx + 1, dtype=np.float64) / float(nx) * Lx
        j = np.arange(ny + 1, dtype=np.float64)
        y = 0.5 * Ly * np.tanh(stretch * (2.0 * j / float(ny) - 1.0)) / np.tanh(stretch)
        z = np.arange(nz + 1, dtype=np.float64) / float(nz) * Lz - 0.5 * Lz
        self.G = G = Grid(x, y, z, (True, False, True), g)
        self.solve_p, self.solve_v = solve_p, solve_v
        self.rho, self.Ubulk, self.Wbulk = float(rho), float(Ubulk), float(Wbulk)
        self.visc = np.full(G.padded, float(visc))
        self.rho_face = np.full(G.padded, self.rho)
        self.opr = laplacian(G)
        self.dtmax, self.cflmax, self.itmax = dtmax, cflmax, itmax
        self.dt, self.t, self.n = dtmax, 0.0, 0
        vel = np.sqrt(Ubulk ** 2 + Wbulk ** 2)
        zm = extended_centres(z, g)[:, None, None]
        xm = extended_centres(x, g)[None, None, :]
        one = np.ones(G.padded)
        self.U = np.where(face_mask(G, 0), 0.0, Ubulk * one)
        self.U = np.where(face_mask(G, 0), self.U, self.U + amp * vel * np.cos(8.0 * 2.0 * np.pi * zm / Lz))
        self.V = np.zeros(G.padded)
        self.W = np.where(face_mask(G, 2), 0.0, Wbulk * one)
        self.W = np.where(face_mask(G, 2), self.W, self.W + amp * vel * np.cos(8.0 * 2.0 * np.pi * xm / Lx))
        self.P = np.zeros(G.padded)

    def _fill(self, inner):
        a = np.zeros(self.G.padded)
        self.G.interior(a)[...] = inner
        return self.G.sync(a)

    def step(self):
        G = self.G
        s = flow_stats(G, self.U, self.V, self.W, self.visc, self.rho, self.dt)
        cfl = s[:6].max()
        dtold = self.dt
        if cfl > 0.0:
            self.dt = min(dtold * self.cflmax / cfl, self.dtmax)
        if self.dt > dtold:
            self.dt = 0.7 * self.dt + (1.0 - 0.7) * dtold
        self.t += self.dt
        self.n += 1
        dt, rho = self.dt, self.rho
        Uo, Vo, Wo = self.U.copy(), self.V.copy(), self.W.copy()
        for _ in range(self.itmax):
            self.U, self.V, self.W = midpoint(self.U, Uo), midpoint(self.V, Vo), midpoint(self.W, Wo)
            dU, dV, dW = dmomdt(G, self.U, self.V, self.W, self.P, rho, self.visc)
            su, vu = bulk(G, 0, self.U, Uo)
            sw, vw = bulk(G, 2, self.W, Wo)
            fu = (self.Ubulk, su / vu) if self.forcing else None
            fw = (self.Wbulk, sw / vw) if self.forcing else None
            res = [mom_residual(G, 0, dt, rho, self.U, Uo, dU, fu),
                   mom_residual(G, 1, dt, rho, self.V, Vo, dV),
                   mom_residual(G, 2, dt, rho, self.W, Wo, dW, fw)]
            for c in range(3):   # solve_implicit
                A = implicit_operator(G, c, dt, rho, self.U, self.V, self.W, self.visc)
                res[c] = self._fill(self.solve_v(A, np.ascontiguousarray(G.interior(res[c]))))
            self.U = apply_residual(self.U, Uo, res[0])
            self.V = apply_residual(self.V, Vo, res[1])
            self.W = apply_residual(self.W, Wo, res[2])
            _, rhs = divergence(G, self.U, self.V, self.W, rho=rho, dt=dt)
            sol = self._fill(self.solve_p(np.ascontiguousarray(G.interior(self.opr)),
                                          np.ascontiguousarray(G.interior(rhs))))
            sol, _ = shift_p(G, sol)
            self.U, self.V, self.W, self.P = correct(G, sol, dt, self.U, self.V, self.W, self.P, self.rho_face,
                                                     self.rho_face, self.rho_face)
