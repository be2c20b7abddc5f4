"""Seeded synthetic pressure-Poisson problems of the shapes NGA2's flow solvers hand
to their pressure solver.

The operator is assembled the way the callers assemble it:

* metrics follow ``src/grid/sgrid_class.f90:160-254`` (naive extension of the mesh
  over the overlap, cell centres, ``dxi = 1/dx``, ``dxmi = 1/(xm(i)-xm(i-1))``)
  and ``src/config/config_class.f90:108`` (``vol = dx*dy*dz``);
* the 7-point stencil is ``-vol*div(grad(p)/rho_face)`` as in
  ``src/two_phase/tpns_class.f90:1565-1593`` (``src/constant_density/
  incomp_class.f90:766-785`` with rho = 1), with the stencil order
  ``[0,0,0],[+1,0,0],[-1,0,0],[0,+1,0],[0,-1,0],[0,0,+1],[0,0,-1]``
  (``incomp_class.f90:758-764``);
* wall faces of non-periodic directions carry zero face metrics, the
  ``umask/vmask/wmask = 2`` rule of ``incomp_class.f90:173-230,516-566``;
* the right-hand side is ``-vol*div(u)`` (``incomp_class.f90:1144-1159``).

Arrays use NGA2's Fortran layout with no overlap: the operator is
``opr[k, j, i, st]`` (``opr(st,i,j,k)`` in Fortran), vectors are ``[k, j, i]``.
Every generator takes a seed; the same seed gives the same bits everywhere.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

#: NGA2's 7-point stencil map for the pressure operator (incomp_class.f90:758-764)
STC7 = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]],
                dtype=np.int32)


@dataclasses.dataclass
class Problem:
    """A pressure-Poisson system in NGA2's layout."""
    name: str
    nx: int
    ny: int
    nz: int
    xper: bool
    yper: bool
    zper: bool
    stc: np.ndarray          # (nst, 3) int32
    opr: np.ndarray          # (nz, ny, nx, nst) float64
    rhs: np.ndarray          # (nz, ny, nx) float64
    vol: np.ndarray          # (nz, ny, nx) float64
    seed: int
    info: dict = dataclasses.field(default_factory=dict)

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)


def _axis(x: np.ndarray):
    """Cell sizes and centroid spacings of one direction.

    ``x`` holds the n+1 node positions.  Returns ``(dx, dxi, dxmi)`` where dx/dxi
    cover the interior cells 1..n and dxmi the faces 1..n+1 (sgrid_class.f90:
    168-254, one overlap layer)."""
    n = x.size - 1
    xe = np.empty(n + 3)
    xe[1:n + 2] = x
    xe[0] = xe[1] - (xe[2] - xe[1])
    xe[n + 2] = xe[n + 1] + (xe[n + 1] - xe[n])
    xm = 0.5 * (xe[:-1] + xe[1:])           # xm(0..n+1)
    dx = xe[1:] - xe[:-1]                   # dx(0..n+1)
    dxm = xm[1:] - xm[:-1]                  # dxm(1..n+1)
    return dx[1:n + 1], 1.0 / dx[1:n + 1], 1.0 / dxm


def assemble_operator(xn, yn, zn, per, rho=None):
    """7-point ``-vol*div(grad/rho_face)`` operator.

    ``xn, yn, zn`` are node coordinates, ``per`` the periodicity triple and
    ``rho`` an optional cell-centred density (nz, ny, nx); face densities are the
    arithmetic mean of the two neighbouring cells (periodic wrap where periodic).
    Returns ``(opr, vol)``."""
    nx, ny, nz = xn.size - 1, yn.size - 1, zn.size - 1
    dx, dxi, dxmi = _axis(np.asarray(xn, np.float64))
    dy, dyi, dymi = _axis(np.asarray(yn, np.float64))
    dz, dzi, dzmi = _axis(np.asarray(zn, np.float64))
    # wall faces carry zero metrics (umask/vmask/wmask = 2)
    if not per[0]:
        dxmi = dxmi.copy(); dxmi[0] = 0.0; dxmi[-1] = 0.0
    if not per[1]:
        dymi = dymi.copy(); dymi[0] = 0.0; dymi[-1] = 0.0
    if not per[2]:
        dzmi = dzmi.copy(); dzmi[0] = 0.0; dzmi[-1] = 0.0
    vol = (dx[None, None, :] * dy[None, :, None]) * dz[:, None, None]

    def face_rho(axis, n):
        # rho on faces 1..n+1 along axis (face f sits between cells f-1 and f),
        # the arithmetic mean of the two cells (the staggered rho_U of tpns)
        if rho is None:
            return None
        r = np.moveaxis(rho, axis, -1)
        lo = np.concatenate([r[..., -1:], r], axis=-1)       # cell f-1 (periodic wrap at f=1)
        hi = np.concatenate([r, r[..., :1]], axis=-1)        # cell f
        return np.moveaxis(0.5 * (lo + hi), -1, axis)

    opr = np.empty((nz, ny, nx, 7))
    # x: per-direction east/west contributions (tpns_class.f90:1571-1584)
    rfx = face_rho(2, nx)
    rfy = face_rho(1, ny)
    rfz = face_rho(0, nz)

    def terms(di, dmi_lo, dmi_hi, rf, axis):
        # divp(1)*divu(-1,i+1), divp(0)*divu(0,i), divp(1)*divu(0,i+1), divp(0)*divu(-1,i)
        shp = [1, 1, 1]
        shp[axis] = -1
        di = di.reshape(shp); lo = dmi_lo.reshape(shp); hi = dmi_hi.reshape(shp)
        e_diag = di * (-hi)
        w_diag = (-di) * lo
        e_off = di * hi
        w_off = (-di) * (-lo)
        if rf is not None:
            # each face term divided by the face density (tpns_class.f90:1571-1584)
            sl_hi = [slice(None)] * 3; sl_hi[axis] = slice(1, None)
            sl_lo = [slice(None)] * 3; sl_lo[axis] = slice(0, -1)
            rhi, rlo = rf[tuple(sl_hi)], rf[tuple(sl_lo)]
            e_diag = e_diag / rhi; w_diag = w_diag / rlo
            e_off = e_off / rhi; w_off = w_off / rlo
        return e_diag, w_diag, e_off, w_off

    xe, xw, xo_e, xo_w = terms(dxi, dxmi[:-1], dxmi[1:], rfx, 2)
    ye, yw, yo_e, yo_w = terms(dyi, dymi[:-1], dymi[1:], rfy, 1)
    ze, zw, zo_e, zo_w = terms(dzi, dzmi[:-1], dzmi[1:], rfz, 0)
    full = (nz, ny, nx)
    opr[..., 0] = np.broadcast_to(((((xe + xw) + ye) + yw) + ze) + zw, full)
    opr[..., 1] = np.broadcast_to(xo_e, full)
    opr[..., 2] = np.broadcast_to(xo_w, full)
    opr[..., 3] = np.broadcast_to(yo_e, full)
    opr[..., 4] = np.broadcast_to(yo_w, full)
    opr[..., 5] = np.broadcast_to(zo_e, full)
    opr[..., 6] = np.broadcast_to(zo_w, full)
    opr *= -vol[..., None]
    # -0.0 where a wall face zeroes a coefficient; keep +0.0 like the Fortran
    opr += 0.0
    return opr, vol


def divergence(U, V, W, xn, yn, zn):
    """FV divergence of face velocities (incomp_class.f90:1144-1159).

    ``U`` is (nz, ny, nx+1) on x-faces 1..nx+1, similarly V and W."""
    dx, dxi, _ = _axis(xn)
    dy, dyi, _ = _axis(yn)
    dz, dzi, _ = _axis(zn)
    return ((-dxi[None, None, :] * U[:, :, :-1] + dxi[None, None, :] * U[:, :, 1:])
            + (-dyi[None, :, None] * V[:, :-1, :] + dyi[None, :, None] * V[:, 1:, :])
            + (-dzi[:, None, None] * W[:-1, :, :] + dzi[:, None, None] * W[1:, :, :]))


def _solenoidal_faces(rng, xn, yn, zn, nmodes=16, kmax=8, Ls=(1.0, 1.0, 1.0)):
    """Face velocities u = curl(A), A = sum_m a_m cos(2 pi k_m.x/L + phi_m).

    Each mode's curl is -sin(theta) (2 pi k/L x a); the sine is evaluated as a
    separable product of 1-D complex exponentials."""
    nx, ny, nz = xn.size - 1, yn.size - 1, zn.size - 1
    xm = 0.5 * (xn[:-1] + xn[1:]); ym = 0.5 * (yn[:-1] + yn[1:]); zm = 0.5 * (zn[:-1] + zn[1:])
    U = np.zeros((nz, ny, nx + 1)); V = np.zeros((nz, ny + 1, nx)); W = np.zeros((nz + 1, ny, nx))
    for _ in range(nmodes):
        k = rng.integers(-kmax, kmax + 1, size=3)
        while not k.any():
            k = rng.integers(-kmax, kmax + 1, size=3)
        a = rng.standard_normal(3)
        phi = rng.uniform(0.0, 2.0 * math.pi)
        kw = 2.0 * math.pi * k / np.asarray(Ls)
        c = -np.cross(kw, a)  # curl(a cos th) = -sin(th) (kw x a)

        def sin_th(x, y, z):
            ex = np.exp(1j * kw[0] * x); ey = np.exp(1j * kw[1] * y); ez = np.exp(1j * kw[2] * z)
            return (np.exp(1j * phi) * ez[:, None, None] * ey[None, :, None] * ex[None, None, :]).imag

        U += c[0] * sin_th(xn, ym, zm)
        V += c[1] * sin_th(xm, yn, zm)
        W += c[2] * sin_th(xm, ym, zn)
    return U, V, W


def uniform_nodes(n, L=1.0, x0=0.0):
    return x0 + np.arange(n + 1, dtype=np.float64) * (L / n)


def periodic_poisson(n=64, seed=0, nmodes=32, kmax=8):
    """Triply periodic constant-coefficient 7-point Laplacian on the unit cube;
    RHS = seeded sum of ``nmodes`` Fourier modes with wavenumbers 1..kmax (random
    sign), N(0,1) amplitudes and uniform phases at cell centres, mean removed."""
    rng = np.random.default_rng(seed)
    xn = uniform_nodes(n)
    opr, vol = assemble_operator(xn, xn, xn, (True, True, True))
    xc = 0.5 * (xn[:-1] + xn[1:])
    rhs = np.zeros((n, n, n))
    for _ in range(nmodes):
        k = rng.integers(1, kmax + 1, size=3) * rng.choice([-1, 1], size=3)
        a = rng.standard_normal()
        phi = rng.uniform(0.0, 2.0 * math.pi)
        ex = np.exp(2j * math.pi * k[0] * xc); ey = np.exp(2j * math.pi * k[1] * xc)
        ez = np.exp(2j * math.pi * k[2] * xc)
        rhs += a * (np.exp(1j * phi) * ez[:, None, None] * ey[None, :, None] * ex[None, None, :]).real
    rhs -= rhs.mean()
    return Problem("periodic_const", n, n, n, True, True, True, STC7.copy(), opr, rhs, vol, seed,
                   {"dx": 1.0 / n, "modes": nmodes, "kmax": kmax})


def drop_density(n, ndrops, rmin, rmax, ratio, rng, per=(True, False, True), width=1.5):
    """Cell-centred density 1 + (ratio-1) H, H = max over drops of
    0.5 (1 - tanh((|x - c| - R)/(width dx))) with periodic distances where periodic."""
    dx = 1.0 / n
    xc = (np.arange(n) + 0.5) * dx
    H = np.zeros((n, n, n))
    centres = rng.uniform(0.0, 1.0, size=(ndrops, 3))
    radii = rng.uniform(rmin, rmax, size=ndrops) * dx
    # tanh(z) rounds to 1 beyond z ~ 19, so each drop only touches a box
    reach = radii + 20.0 * width * dx
    for c, R, rr in zip(centres, radii, reach):
        idx = []
        dists = []
        for d in range(3):
            lo = int(math.floor((c[d] - rr) / dx)) - 1
            hi = int(math.ceil((c[d] + rr) / dx)) + 1
            ii = np.arange(lo, hi + 1)
            if per[d]:
                ii = np.unique(np.mod(ii, n))
            else:
                ii = ii[(ii >= 0) & (ii < n)]
            dd = xc[ii] - c[d]
            if per[d]:
                dd = dd - np.round(dd)
            idx.append(ii)
            dists.append(dd)
        r = np.sqrt(dists[0][None, None, :] ** 2 + dists[1][None, :, None] ** 2 + dists[2][:, None, None] ** 2)
        h = 0.5 * (1.0 - np.tanh((r - R) / (width * dx)))
        sub = np.ix_(idx[2], idx[1], idx[0])
        H[sub] = np.maximum(H[sub], h)
    return 1.0 + (ratio - 1.0) * H, centres, radii


def drops_poisson(n=256, seed=0, ndrops=48, rmin=6.0, rmax=20.0, ratio=1000.0, noise=0.01,
                  per=(True, False, True)):
    """Variable-density pressure Poisson: rho = ratio inside seeded drops, 1 outside,
    tanh-smeared over 1.5 cells; walls (Neumann) in the non-periodic directions;
    RHS = -vol div(u), u = curl of a seeded random vector potential plus N(0, noise)
    face noise, wall-normal velocity zero at walls, mean removed."""
    rng = np.random.default_rng(seed)
    rho, centres, radii = drop_density(n, ndrops, rmin, rmax, ratio, rng, per)
    xn = uniform_nodes(n)
    opr, vol = assemble_operator(xn, xn, xn, per, rho=rho)
    U, V, W = _solenoidal_faces(rng, xn, xn, xn)
    U += noise * rng.standard_normal(U.shape)
    V += noise * rng.standard_normal(V.shape)
    W += noise * rng.standard_normal(W.shape)
    if per[0]:
        U[:, :, -1] = U[:, :, 0]
    else:
        U[:, :, 0] = 0.0; U[:, :, -1] = 0.0
    if per[1]:
        V[:, -1, :] = V[:, 0, :]
    else:
        V[:, 0, :] = 0.0; V[:, -1, :] = 0.0
    if per[2]:
        W[-1, :, :] = W[0, :, :]
    else:
        W[0, :, :] = 0.0; W[-1, :, :] = 0.0
    rhs = -vol * divergence(U, V, W, xn, xn, xn)
    rhs -= rhs.mean()
    return Problem("drops_varcoeff", n, n, n, per[0], per[1], per[2], STC7.copy(), opr, rhs, vol, seed,
                   {"ndrops": ndrops, "radii_cells": [rmin, rmax], "rho_ratio": ratio,
                    "rho_min": float(rho.min()), "rho_max": float(rho.max())})


def helmholtz_mast(n=256, seed=0, ndrops=48, rmin=6.0, rmax=20.0, L=1e-2, rho_l=1000.0, rho_g=1.0,
                   c_l=1500.0, c_g=340.0, u_ref=1.0, cfl=0.5, p0=1.0e5, sigma=0.07, noise=0.01,
                   per=(True, False, True)):
    """Pressure Helmholtz system of the compressible two-phase solver mast
    (``src/two_phase/mast_class.f90:3900-3960``, ``update_Helmholtz_LHS/RHS``):

        opr = -dt^2 div(grad(.)/rho_face) + 1/RHOSS2        (no volume factor)
        rhs = (PA - P)/RHOSS2 - dt div(u)                    (P = 0: first sub-iteration)

    with the mixture bulk modulus of ``mast_class.f90:3494-3499`` away from
    interface models, RHOSS2 = 1/(VF/(rho_l c_l^2) + (1-VF)/(rho_g c_g^2)).
    Liquid drops (VF = 1, water-like) in gas (VF = 0, air-like), tanh-smeared
    over 1.5 cells, in a box of side ``L`` metres; dt = cfl dx/u_ref (a
    convective time step, so the acoustic CFL is c dt/dx >> 1 and the system is
    a Poisson problem shifted by a small positive diagonal: nonsingular);
    u = u_ref curl(A) + N(0, noise u_ref) at the faces, wall-normal velocity zero
    at walls; PA = p0 + the Laplace jump 2 sigma/R inside each drop + 1e-3 p0
    N(0, 1) noise.  The 7-point stencil order is NGA2's."""
    rng = np.random.default_rng(seed)
    ratio = rho_l / rho_g
    rho1, centres, radii = drop_density(n, ndrops, rmin, rmax, ratio, rng, per)
    vf = (rho1 - 1.0) / (ratio - 1.0)
    rho = rho_g * rho1
    inv_rhoss2 = vf / (rho_l * c_l * c_l) + (1.0 - vf) / (rho_g * c_g * c_g)
    xn = uniform_nodes(n, L)
    lap, vol = assemble_operator(xn, xn, xn, per, rho=rho)  # -vol div(grad/rho_face)
    dx = L / n
    dt = cfl * dx / u_ref
    opr = (dt * dt) * (lap / vol[..., None])
    opr[..., 0] += inv_rhoss2
    U, V, W = _solenoidal_faces(rng, xn, xn, xn, Ls=(L, L, L))
    scale = u_ref / max(np.abs(U).max(), np.abs(V).max(), np.abs(W).max())
    U = scale * U + noise * u_ref * rng.standard_normal(U.shape)
    V = scale * V + noise * u_ref * rng.standard_normal(V.shape)
    W = scale * W + noise * u_ref * rng.standard_normal(W.shape)
    if per[0]:
        U[:, :, -1] = U[:, :, 0]
    else:
        U[:, :, 0] = 0.0; U[:, :, -1] = 0.0
    if per[1]:
        V[:, -1, :] = V[:, 0, :]
    else:
        V[:, 0, :] = 0.0; V[:, -1, :] = 0.0
    if per[2]:
        W[-1, :, :] = W[0, :, :]
    else:
        W[0, :, :] = 0.0; W[-1, :, :] = 0.0
    jump = 2.0 * sigma / float(np.mean(radii * L))
    PA = p0 + jump * vf + 1e-3 * p0 * rng.standard_normal(vf.shape)
    rhs = PA * inv_rhoss2 - dt * divergence(U, V, W, xn, xn, xn)
    return Problem("helmholtz_mast", n, n, n, per[0], per[1], per[2], STC7.copy(), opr, rhs, vol, seed,
                   {"ndrops": ndrops, "radii_cells": [rmin, rmax], "L": L, "dt": dt,
                    "acoustic_cfl": [c_l * dt / dx, c_g * dt / dx], "rho": [rho_l, rho_g],
                    "c": [c_l, c_g]})


def channel_poisson(nx=512, ny=512, nz=512, seed=0, stretch=2.0, Lx=2.0 * math.pi, Ly=2.0,
                    Lz=2.0 * math.pi, noise=0.1):
    """Stretched-grid channel: periodic x/z, walls in y with
    y_j = Ly/2 tanh(s(2(j-1)/ny - 1))/tanh(s) (examples/channel/src/geometry.f90:37-39);
    constant density; RHS = -vol div(u), u = laminar parabolic profile in x plus
    N(0, noise) face perturbations, zero wall-normal velocity at the walls."""
    rng = np.random.default_rng(seed)
    xn = uniform_nodes(nx, Lx)
    zn = uniform_nodes(nz, Lz)
    j = np.arange(ny + 1, dtype=np.float64)
    yn = 0.5 * Ly * np.tanh(stretch * (2.0 * j / ny - 1.0)) / math.tanh(stretch)
    opr, vol = assemble_operator(xn, yn, zn, (True, False, True))
    ym = 0.5 * (yn[:-1] + yn[1:])
    h = 0.5 * Ly
    U = np.broadcast_to((1.0 - (ym / h) ** 2)[None, :, None], (nz, ny, nx + 1)).copy()
    U += noise * rng.standard_normal(U.shape)
    V = noise * rng.standard_normal((nz, ny + 1, nx))
    W = noise * rng.standard_normal((nz + 1, ny, nx))
    U[:, :, -1] = U[:, :, 0]
    W[-1, :, :] = W[0, :, :]
    V[:, 0, :] = 0.0; V[:, -1, :] = 0.0
    rhs = -vol * divergence(U, V, W, xn, yn, zn)
    rhs -= rhs.mean()
    return Problem("channel_stretched", nx, ny, nz, True, False, True, STC7.copy(), opr, rhs, vol, seed,
                   {"stretch": stretch, "first_cell_over_h": float((yn[1] - yn[0]) / h),
                    "L": [Lx, Ly, Lz]})


def random_operator(nx, ny, nz, per, seed=0, full27=False, diag_boost=0.0, asym=0.0):
    """Random diagonally dominant (or singular with zero row sums when
    ``diag_boost == 0``) operator for property tests: symmetric 7-point from
    random positive face conductances, optionally with random 27-point
    off-diagonal couplings (non-symmetric), or with the 7-point off-diagonals
    scaled by 1 + asym*U(0,1) (non-symmetric 7-point)."""
    rng = np.random.default_rng(seed)
    xn = uniform_nodes(nx); yn = uniform_nodes(ny); zn = uniform_nodes(nz)
    rho = np.exp(rng.uniform(-2.0, 2.0, size=(nz, ny, nx)))
    opr7, vol = assemble_operator(xn, yn, zn, per, rho=rho)
    if diag_boost:
        opr7[..., 0] += diag_boost * np.abs(opr7[..., 0])
    if asym:
        opr7[..., 1:] *= 1.0 + asym * rng.uniform(0.0, 1.0, size=opr7[..., 1:].shape)
    if not full27:
        return STC7.copy(), opr7
    stc = np.array([[i, j, k] for k in (-1, 0, 1) for j in (-1, 0, 1) for i in (-1, 0, 1)], dtype=np.int32)
    opr = np.zeros((nz, ny, nx, 27))
    scale = np.abs(opr7[..., 1:]).mean()
    extra = -0.05 * scale * rng.uniform(0.0, 1.0, size=(nz, ny, nx, 27))
    for st, s in enumerate(stc):
        if abs(s).sum() >= 2:
            opr[..., st] = extra[..., st]
    for st7, s7 in enumerate(STC7):
        q = int(np.where((stc == s7).all(axis=1))[0][0])
        opr[..., q] += opr7[..., st7]
    # keep the row sum of the added couplings on the diagonal
    opr[..., 13] -= extra[..., [st for st, s in enumerate(stc) if abs(s).sum() >= 2]].sum(axis=-1)
    return stc, opr


def remove_mean(p, vol=None):
    """Volume-weighted mean removal (shift_p, incomp_class.f90:1720-1740, VF = 1)."""
    if vol is None:
        return p - p.mean()
    return p - (p * vol).sum() / vol.sum()
