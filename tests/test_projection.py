"""The steps of the time loop around the pressure solve (include/nga_projection.h):
operator assembly, divergence and right-hand side, shift_p, get_pgrad, the
velocity correction, get_dmomdt and solve_implicit's operator.

CPU: the library exports every declared symbol; the numpy oracle
(oracle/projection_oracle.py) agrees with the problem generators' operator and
divergence, a whole projection through the oracle leaves a divergence-free
velocity, its get_dmomdt converges at second order on a Taylor-Green field and
gives the one-sided wall values on a Poiseuille profile, and its implicit
operator equals rho - dt/2 (viscous get_dmomdt) and the linearised convective
get_dmomdt to round-off.  GPU: every kernel equals the oracle bit for bit
(shift_p's mean to round-off), periodic and with walls, and a projection
chained entirely on the device (assembly -> setup -> divergence -> solve ->
shift -> correction) leaves a divergence-free velocity.
"""
import math
import os
import re

import numpy as np
import pytest

from nga2_b200 import problems as P
from oracle import projection_oracle as PO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "nga_projection.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(nga_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_projection_symbol():
    from nga2_b200 import bbmg as B
    from nga2_b200 import projection as PR
    lib = B.load()
    names = header_functions()
    assert len(names) == 16
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(PR.EXPORTS) == names
    PR.lib()  # every signature binds


def stretched(n, L=1.0, s=1.5):
    j = np.arange(n + 1, dtype=np.float64)
    return 0.5 * L * (1.0 + np.tanh(s * (2.0 * j / n - 1.0)) / math.tanh(s))


def make_fields(G, rng, rho_cells=None):
    """Padded random velocities, face densities (arithmetic means of the
    cells, the generators' rule) and pressure; ghosts random as well."""
    shp = G.padded
    U, V, W, Pr = (rng.standard_normal(shp) for _ in range(4))
    if rho_cells is None:
        rho_cells = np.exp(rng.uniform(-2.0, 2.0, size=(G.nz, G.ny, G.nx)))
    rc = np.ones(shp)
    G.interior(rc)[...] = rho_cells
    rc = G.sync(rc)
    g = G.g
    # non-periodic overlap cells: copy the adjacent interior layer
    if not G.per[0]:
        rc[:, :, :g] = rc[:, :, g:g + 1]; rc[:, :, G.nx + g:] = rc[:, :, G.nx + g - 1:G.nx + g]
    if not G.per[1]:
        rc[:, :g, :] = rc[:, g:g + 1, :]; rc[:, G.ny + g:, :] = rc[:, G.ny + g - 1:G.ny + g, :]
    if not G.per[2]:
        rc[:g] = rc[g:g + 1]; rc[G.nz + g:] = rc[G.nz + g - 1:G.nz + g]
    rU, rV, rW = np.ones(shp), np.ones(shp), np.ones(shp)
    rU[:, :, 1:] = 0.5 * (rc[:, :, :-1] + rc[:, :, 1:])
    rV[:, 1:, :] = 0.5 * (rc[:, :-1, :] + rc[:, 1:, :])
    rW[1:, :, :] = 0.5 * (rc[:-1, :, :] + rc[1:, :, :])
    return U, V, W, Pr, (rU, rV, rW), rho_cells


def test_oracle_laplacian_matches_generator():
    """update_laplacian with arithmetic-mean face densities is the generators'
    -vol div(grad/rho_face) operator, bit for bit."""
    for per, g in (((True, False, True), 1), ((False, False, False), 2), ((True, True, True), 1)):
        xn, yn, zn = P.uniform_nodes(12), stretched(10), P.uniform_nodes(9, 2.0)
        G = PO.Grid(xn, yn, zn, per, g)
        rng = np.random.default_rng(1)
        *_, rho, rho_c = make_fields(G, rng)
        opr = PO.laplacian(G, *rho)
        ref, vol = P.assemble_operator(xn, yn, zn, per, rho=rho_c)
        assert np.array_equal(G.interior(opr), ref)
        assert np.array_equal(G.vol, vol)


def test_oracle_divergence_matches_generator():
    xn, yn, zn = P.uniform_nodes(12), stretched(10), P.uniform_nodes(9, 2.0)
    G = PO.Grid(xn, yn, zn, (True, False, True), 1)
    rng = np.random.default_rng(2)
    U, V, W, *_ = make_fields(G, rng)
    div, rhs = PO.divergence(G, U, V, W, dt=0.1)
    g = G.g
    Uf = U[g:-g, g:-g, g:g + G.nx + 1]
    Vf = V[g:-g, g:g + G.ny + 1, g:-g]
    Wf = W[g:g + G.nz + 1, g:-g, g:-g]
    assert np.array_equal(G.interior(div), P.divergence(Uf, Vf, Wf, xn, yn, zn))
    assert np.array_equal(G.interior(rhs), -((G.vol * G.interior(div)) * 1.0) / 0.1)


def projection_oracle_chain(n=16, per=(True, False, True), seed=3):
    """One projection through the oracle: assemble, solve (oracle bbmg),
    shift, correct; returns max|div| before and after."""
    from oracle.oracle import OracleBBMG, PCG_BBOX
    xn = P.uniform_nodes(n)
    G = PO.Grid(xn, xn, xn, per, 1)
    rng = np.random.default_rng(seed)
    U, V, W, Pr, rho, _ = make_fields(G, rng)
    U, V, W = G.sync(U), G.sync(V), G.sync(W)
    # zero normal velocity on the walls
    g = G.g
    if not per[1]:
        V[:, g, :] = 0.0; V[:, g + n, :] = 0.0
    dt = 0.01
    opr = PO.laplacian(G, *rho)
    div0, rhs = PO.divergence(G, U, V, W, dt=dt)
    rhs_i = G.interior(rhs).copy()
    rhs_i -= rhs_i.mean()
    o = OracleBBMG(n, n, n, *per, method=PCG_BBOX, rcvg=1e-12)
    o.setup(P.STC7, np.ascontiguousarray(G.interior(opr)))
    x, it, rerr = o.solve(rhs_i)
    sol = np.zeros(G.padded)
    G.interior(sol)[...] = x
    sol, mean = PO.shift_p(G, G.sync(sol))
    U1, V1, W1, P1 = PO.correct(G, sol, dt, U, V, W, Pr, *rho)
    div1, _ = PO.divergence(G, U1, V1, W1)
    return np.abs(G.interior(div0)).max(), np.abs(G.interior(div1)).max(), abs(mean)


def test_oracle_projection_removes_divergence():
    d0, d1, _ = projection_oracle_chain()
    assert d1 < 1e-9 * d0, (d0, d1)


# ----------------------------------------------------------------------------- GPU
GCASES = [((12, 10, 9), (True, False, True), 1), ((8, 8, 8), (True, True, True), 2),
          ((9, 7, 6), (False, False, False), 1), ((16, 12, 10), (False, True, True), 2)]
GIDS = ["x".join(map(str, d)) + "-" + "".join("p" if p else "w" for p in per) + f"-g{g}" for d, per, g in GCASES]


def gpu_setup(dims, per, g, seed):
    import torch
    from nga2_b200.projection import Projection
    nx, ny, nz = dims
    xn, yn, zn = P.uniform_nodes(nx), stretched(ny), P.uniform_nodes(nz, 2.0)
    G = PO.Grid(xn, yn, zn, per, g)
    pr = Projection(xn, yn, zn, *per, ghost=g, device=0)
    rng = np.random.default_rng(seed)
    U, V, W, Pr, rho, _ = make_fields(G, rng)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return G, pr, (U, V, W, Pr, rho), T


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per,g", GCASES, ids=GIDS)
def test_laplacian_bitexact(dims, per, g):
    G, pr, (U, V, W, Pr, rho), T = gpu_setup(dims, per, g, 1)
    for r in (rho, (None, None, None)):
        ref = PO.laplacian(G, *r)
        opr = pr.update_laplacian(*(None if a is None else T(a) for a in r)).cpu().numpy()
        assert np.array_equal(G.interior(opr), G.interior(ref))
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per,g", GCASES, ids=GIDS)
def test_divergence_and_rhs_bitexact(dims, per, g):
    G, pr, (U, V, W, Pr, rho), T = gpu_setup(dims, per, g, 2)
    rng = np.random.default_rng(9)
    div0 = rng.standard_normal(G.padded)
    for rho_s, dt in ((1.0, 0.01), (1000.0, 3e-4)):
        ref_div, ref_rhs = PO.divergence(G, U, V, W, rho=rho_s, dt=dt, div_out=div0)
        div, rhs = pr.get_div(T(U), T(V), T(W), rho=rho_s, dt=dt, div=T(div0))
        assert np.array_equal(div.cpu().numpy(), ref_div)
        assert np.array_equal(G.interior(rhs.cpu().numpy()), G.interior(ref_rhs))
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per,g", GCASES, ids=GIDS)
def test_pgrad_and_correct_bitexact(dims, per, g):
    G, pr, (U, V, W, Pr, rho), T = gpu_setup(dims, per, g, 3)
    rng = np.random.default_rng(4)
    S = G.sync(rng.standard_normal(G.padded))
    gref = PO.pgrad(G, S)
    z = lambda: T(rng.standard_normal(G.padded))
    gx, gy, gz = pr.get_pgrad(T(S), z(), z(), z())
    for a, b in zip((gx, gy, gz), gref):
        # ghosts outside walls are left as the caller had them
        assert np.array_equal(G.interior(a.cpu().numpy()), G.interior(b))
    U1, V1, W1, P1 = PO.correct(G, S, 0.02, U, V, W, Pr, *rho)
    tU, tV, tW, tP = T(U), T(V), T(W), T(Pr)
    pr.correct(T(S), 0.02, tU, tV, tW, tP, *(T(r) for r in rho))
    for a, b in zip((tU, tV, tW, tP), (U1, V1, W1, P1)):
        assert np.array_equal(a.cpu().numpy(), b)
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per,g", GCASES, ids=GIDS)
def test_shift_p(dims, per, g):
    G, pr, (U, V, W, Pr, rho), T = gpu_setup(dims, per, g, 5)
    Pr = Pr + 3.0
    ref, mref = PO.shift_p(G, Pr)
    t = T(Pr)
    m = pr.shift_p(t)
    assert abs(m - mref) <= 1e-14 * abs(mref)
    out = t.cpu().numpy()
    assert np.abs(out - ref).max() <= 1e-14 * np.abs(ref).max()
    # outside walls the overlap is untouched; the periodic overlap holds images
    assert np.array_equal(out, G.sync(out))
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_projection_on_device_removes_divergence(precision):
    """Assembly -> bbmg_setup on the device operator -> divergence and rhs ->
    solve -> shift_p -> correction, all on device arrays: the corrected
    velocity is discretely divergence-free, and the chain matches the oracle's."""
    import torch
    from nga2_b200.bbmg import BBMG, FP64, MIXED, PCG_BBOX
    from nga2_b200.projection import Projection
    n, per, g = 32, (True, False, True), 1
    xn = P.uniform_nodes(n)
    G = PO.Grid(xn, xn, xn, per, g)
    rng = np.random.default_rng(7)
    rho_c, _, _ = P.drop_density(n, 4, 2.0, 5.0, 1000.0, rng, per)
    U, V, W, Pr, rho, _ = make_fields(G, rng, rho_cells=rho_c)
    U, V, W = G.sync(U), G.sync(V), G.sync(W)
    V[:, g, :] = 0.0; V[:, g + n, :] = 0.0
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pr = Projection(xn, xn, xn, *per, ghost=g, device=0)
    tU, tV, tW, tP = T(U), T(V), T(W), T(Pr)
    trho = tuple(T(r) for r in rho)
    dt = 1e-3
    opr = pr.update_laplacian(*trho)
    h = BBMG(n, n, n, *per, ghost=g, method=PCG_BBOX, precision=FP64 if precision == "fp64" else MIXED,
             rcvg=1e-11, device=0)
    h.setup(P.STC7, opr)
    div0, rhs = pr.get_div(tU, tV, tW, dt=dt)
    sol = torch.zeros_like(rhs)
    _, it, rerr, st = h.solve(rhs, sol)
    assert st == 0
    pr.shift_p(sol)
    pr.correct(sol, dt, tU, tV, tW, tP, *trho)
    div1, _ = pr.get_div(tU, tV, tW)
    d0 = G.interior(div0.cpu().numpy())
    d1 = G.interior(div1.cpu().numpy())
    assert np.abs(d1).max() < 1e-8 * np.abs(d0).max(), (np.abs(d1).max(), np.abs(d0).max())
    h.close()
    pr.close()


# ----------------------------------------------------------------------------- momentum right-hand side
def taylor_green(n, rho=1.3, mu=0.02):
    """Fields of u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 and
    p = cos x sin z on the faces / centres of a uniform periodic (2 pi)^3
    grid, with the exact time derivatives of rho u, rho v, rho w there:
    -rho/2 sin 2x cos^2 z - 3 mu u + sin x sin z, -rho/2 sin 2y cos^2 z - 3 mu v,
    -cos x cos z."""
    xn = P.uniform_nodes(n, 2.0 * math.pi)
    G = PO.Grid(xn, xn, xn, (True, True, True), 1)
    h = 2.0 * math.pi / n
    idx = np.arange(-1, n + 1, dtype=np.float64)
    f, c = idx * h, (idx + 0.5) * h     # face and centre coordinates of padded index 0 .. n+1
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    Zf, Yf, Xf = np.meshgrid(f, f, f, indexing="ij")
    U = np.sin(Xf) * np.cos(Y) * np.cos(Z)
    V = -np.cos(X) * np.sin(Yf) * np.cos(Z)
    W = np.zeros(G.padded)
    Pr = np.cos(X) * np.sin(Z)
    exact = (-0.5 * rho * np.sin(2 * Xf) * np.cos(Z) ** 2 - 3.0 * mu * U + np.sin(Xf) * np.sin(Z),
             -0.5 * rho * np.sin(2 * Yf) * np.cos(Z) ** 2 - 3.0 * mu * V,
             -np.cos(X) * np.cos(Zf))
    return G, (U, V, W, Pr), exact, np.full(G.padded, mu)


def test_oracle_dmomdt_converges_on_taylor_green():
    """The oracle's get_dmomdt is second-order accurate on a smooth periodic
    field, and the flux form conserves momentum to round-off."""
    rho = 1.3
    errs = []
    for n in (16, 32):
        G, (U, V, W, Pr), exact, visc = taylor_green(n, rho)
        out = PO.dmomdt(G, U, V, W, Pr, rho, visc)
        e = max(np.abs(G.interior(o) - G.interior(x)).max() for o, x in zip(out, exact))
        errs.append(e / max(np.abs(G.interior(x)).max() for x in exact))
        for o in out:
            assert abs(G.interior(o).sum()) < 1e-10 * np.abs(G.interior(o)).sum()
    assert errs[0] < 0.05 and errs[1] < errs[0] / 3.5, errs


PCASES = [((12, 10, 9), (True, True, True), 1), ((8, 8, 8), (True, True, True), 2),
          ((16, 12, 10), (True, True, True), 2), ((5, 17, 6), (True, True, True), 1),
          ((12, 10, 9), (True, False, True), 1), ((8, 8, 8), (False, False, False), 2),
          ((16, 12, 10), (False, True, True), 1), ((6, 9, 7), (True, True, False), 2)]
PIDS = ["x".join(map(str, d)) + "-" + "".join("p" if p else "w" for p in per) + f"-g{g}" for d, per, g in PCASES]


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per,g", PCASES, ids=PIDS)
def test_dmomdt_bitexact(dims, per, g):
    """k_dmomdt equals the oracle's get_dmomdt bit for bit on stretched grids,
    periodic or with walls, with a viscosity array and with a constant
    viscosity (random values in every overlap and wall cell)."""
    G, pr, (U, V, W, Pr, _), T = gpu_setup(dims, per, g, 11)
    U, V, W, Pr = (G.sync(a) for a in (U, V, W, Pr))
    rng = np.random.default_rng(12)
    visc = G.sync(np.exp(rng.uniform(-7.0, -3.0, size=G.padded)))
    tU, tV, tW, tP = T(U), T(V), T(W), T(Pr)
    for rho, vis, v0 in ((1.0, visc, 0.0), (998.2, None, 1.3e-3)):
        ref = PO.dmomdt(G, U, V, W, Pr, rho, vis if vis is not None else np.full(G.padded, v0))
        out = pr.get_dmomdt(tU, tV, tW, tP, rho=rho, visc=None if vis is None else T(vis), visc0=v0)
        for a, b in zip(out, ref):
            assert np.array_equal(a.cpu().numpy(), b)
    pr.close()


def test_oracle_dmomdt_walls_poiseuille():
    """A parabolic channel profile between walls in y (zero velocity in the
    wall cells): the viscous term is mu U'' = -8 mu Um exactly in the interior
    rows and -6 mu Um in the rows next to the walls, where the wall gradient
    is NGA2's one-sided (U(0) - U_wall) / (ym(0) - y(0)); the other components'
    derivatives vanish."""
    nx, ny, nz, mu, um, rho = 8, 16, 4, 0.02, 1.5, 1.3
    xn, yn, zn = P.uniform_nodes(nx, 2.0), P.uniform_nodes(ny), P.uniform_nodes(nz, 0.5)
    G = PO.Grid(xn, yn, zn, (True, False, True), 1)
    ym = 0.5 * (yn[:-1] + yn[1:])
    U = np.zeros(G.padded)
    G.interior(U)[...] = (4.0 * um * ym * (1.0 - ym))[None, :, None]
    U = G.sync(U)
    Z = np.zeros(G.padded)
    dU, dV, dW = PO.dmomdt(G, U, Z, Z, Z, rho, np.full(G.padded, mu))
    d = G.interior(dU)
    ref = np.full(d.shape, -8.0 * mu * um)
    ref[:, 0, :] = ref[:, -1, :] = -6.0 * mu * um
    assert np.abs(d - ref).max() < 1e-11
    assert np.abs(G.interior(dV)).max() < 1e-12 and np.abs(G.interior(dW)).max() < 1e-12


def apply7(G, opr, x):
    """y = opr x on the interior (NGA2 stencil order, ghost values of x used)."""
    offs = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    y = np.zeros((G.nz, G.ny, G.nx))
    for q, (a, b, c) in enumerate(offs):
        y = y + opr[..., q] * G.interior(x, di=a, dj=b, dk=c)
    return y


@pytest.mark.parametrize("per", [(True, True, True), (True, False, True), (False, True, False)])
def test_oracle_implicit_operator_viscous_part_is_dmomdt(per):
    """With no base velocity the operator solve_implicit assembles is
    rho - dt/2 L_visc, and L_visc x is get_dmomdt of the field x (the other
    components zero, no pressure): the two restatements agree to round-off on
    a stretched grid with a variable viscosity, walls included."""
    nx, ny, nz = 9, 10, 8
    xn, yn, zn = stretched(nx), P.uniform_nodes(ny, 2.0), stretched(nz, 0.5, 1.2)
    G = PO.Grid(xn, yn, zn, per, 1)
    rng = np.random.default_rng(21)
    visc = G.sync(np.exp(rng.uniform(-4.0, -2.0, size=G.padded)))
    Z = np.zeros(G.padded)
    dt, rho = 0.3, 1.7
    for c in range(3):
        x = np.zeros(G.padded)
        G.interior(x)[...] = rng.standard_normal((nz, ny, nx))
        x = G.sync(x)
        if not per[c]:  # the component's wall face holds the no-slip value
            sl = [slice(None)] * 3
            sl[2 - c] = G.g
            x[tuple(sl)] = 0.0
        opr = PO.implicit_operator(G, c, dt, rho, Z, Z, Z, visc)
        fields = [Z, Z, Z]
        fields[c] = x
        d = PO.dmomdt(G, *fields, Z, 0.0, visc)[c]
        ref = rho * G.interior(x) - 0.5 * dt * G.interior(d)
        got = apply7(G, opr, x)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), c


def wall_zero(G, a, comp):
    """Zero the overlap layers of non-periodic directions and, for the
    component normal to a wall, its wall face (NGA2's no-slip values)."""
    g = G.g
    for d in range(3):
        if G.per[d]:
            continue
        ax = 2 - d
        n = (G.nx, G.ny, G.nz)[d]
        sl = [slice(None)] * 3
        sl[ax] = slice(0, g)
        a[tuple(sl)] = 0.0
        sl[ax] = slice(g + n, None)
        a[tuple(sl)] = 0.0
        if d == comp:
            sl[ax] = g
            a[tuple(sl)] = 0.0
    return a


@pytest.mark.parametrize("per", [(True, True, True), (True, False, True), (False, False, True)])
def test_oracle_implicit_operator_convective_part_is_linearised_dmomdt(per):
    """Without viscosity the operator applied to the base velocity's own
    component u is the linearisation of the convective fluxes: rho u - dt/2
    (2 N + T) = rho u - dt/2 (N + D), with N the part of get_dmomdt's
    convective derivative from u alone (quadratic in u, hence the 2) and D
    the whole of it."""
    nx, ny, nz = 8, 9, 10
    xn, yn, zn = stretched(nx), P.uniform_nodes(ny, 2.0), stretched(nz, 0.5, 1.2)
    G = PO.Grid(xn, yn, zn, per, 1)
    rng = np.random.default_rng(22)
    Z = np.zeros(G.padded)
    vel = []
    for c in range(3):
        a = np.zeros(G.padded)
        G.interior(a)[...] = rng.standard_normal((nz, ny, nx))
        vel.append(wall_zero(G, G.sync(a), c))
    dt, rho = 0.2, 1.3
    for c in range(3):
        opr = PO.implicit_operator(G, c, dt, rho, *vel, Z)
        only = [Z, Z, Z]
        only[c] = vel[c]
        N = G.interior(PO.dmomdt(G, *only, Z, rho, Z)[c])
        D = G.interior(PO.dmomdt(G, *vel, Z, rho, Z)[c])
        ref = rho * G.interior(vel[c]) - 0.5 * dt * (N + D)
        got = apply7(G, opr, vel[c])
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), c


ICASES = [((12, 10, 9), (True, True, True), 1), ((10, 12, 8), (True, False, True), 1),
          ((8, 9, 10), (False, False, True), 2), ((9, 8, 8), (False, False, False), 1)]
IIDS = ["x".join(map(str, d)) + "-" + "".join("p" if p else "w" for p in per) + f"-g{g}" for d, per, g in ICASES]


@pytest.mark.gpu
@pytest.mark.parametrize("dims,per,g", ICASES, ids=IIDS)
def test_implicit_operator_bitexact(dims, per, g):
    """k_implicit_opr equals the oracle's solve_implicit operator bit for bit
    on the interior, for the three components, with a viscosity array and a
    constant viscosity."""
    G, pr, (U, V, W, Pr, _), T = gpu_setup(dims, per, g, 31)
    U, V, W = (G.sync(a) for a in (U, V, W))
    rng = np.random.default_rng(32)
    visc = G.sync(np.exp(rng.uniform(-5.0, -2.0, size=G.padded)))
    tU, tV, tW = T(U), T(V), T(W)
    for vis, v0, rho, dt in ((visc, 0.0, 1.0, 0.01), (None, 2e-3, 998.2, 3e-4)):
        for c in range(3):
            ref = PO.implicit_operator(G, c, dt, rho, U, V, W, vis if vis is not None else np.full(G.padded, v0))
            got = pr.implicit_operator(c, dt, rho, tU, tV, tW, visc=None if vis is None else T(vis), visc0=v0)
            got = got.cpu().numpy()[g:g + G.nz, g:g + G.ny, g:g + G.nx]
            assert np.array_equal(got, ref), (c, np.abs(got - ref).max())
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("per", [(True, True, True), (True, False, True)])
def test_solve_implicit_solves_the_operator(per):
    """Incomp.solve_implicit: per component the bbmg multigrid solve of the
    (non-symmetric) operator returns x with |A x - r| <= 1e-9 |r|, A the
    oracle's operator and r the residual it was given."""
    import torch
    from nga2_b200.incomp import Incomp
    nx, ny, nz = 16, 12, 8
    xn, yn, zn = P.uniform_nodes(nx, 2.0), stretched(ny), P.uniform_nodes(nz, 0.5)
    G = PO.Grid(xn, yn, zn, per, 1)
    fs = Incomp(xn, yn, zn, rho=1.2, visc=0.05, per=per, implicit_rcvg=1e-11, implicit_maxit=200)
    rng = np.random.default_rng(33)
    vel, res = [], []
    for c in range(3):
        a = np.zeros(G.padded)
        G.interior(a)[...] = rng.standard_normal((nz, ny, nx))
        vel.append(wall_zero(G, G.sync(a), c))
        r = np.zeros(G.padded)
        G.interior(r)[...] = rng.standard_normal((nz, ny, nx))
        res.append(wall_zero(G, G.sync(r), c))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for dst, src in zip((fs.U, fs.V, fs.W), vel):
        dst.copy_(T(src))
    tres = [T(r) for r in res]
    dt = 0.05
    its = fs.solve_implicit(dt, tres)
    assert all(0 < i < 200 for i in its), its
    visc = np.full(G.padded, 0.05)
    for c in range(3):
        A = PO.implicit_operator(G, c, dt, 1.2, *vel, visc)
        x = tres[c].cpu().numpy()
        r = G.interior(res[c])
        assert np.abs(apply7(G, A, x) - r).max() <= 1e-9 * np.abs(r).max(), c
    fs.close()
