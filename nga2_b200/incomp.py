"""Constant-density incompressible flow on the GPU.

The device counterpart of NGA2's ``incomp`` solver
(src/constant_density/incomp_class.f90) for the calls that its examples make
in their time loops -- the forced homogeneous turbulence example
(examples/hit/src/simulation.f90:256-352, triply periodic, explicit
sub-iterations) and the channel example (examples/channel/src/simulation.f90:
256-340, walls in y, implicit viscous solves) -- with the pressure Poisson
equation and the implicit velocity systems solved by this package's bbmg.
Every field operation runs as a kernel of the projection library
(include/nga_projection.h):

* ``get_dmomdt``                           -> nga_proj_dmomdt
* ``U = 0.5*(U + Uold)``                   -> nga_proj_midpoint
* residual, linear forcing, ``U = 2U - Uold + res/rho`` -> nga_proj_advance
* residual with bulk forcing, ``U = 2U - Uold + res``
                                           -> nga_proj_mom_residual, nga_proj_apply_residual
* ``solve_implicit``                       -> nga_proj_implicit_operator + bbmg (BBMG_BBOX)
* ``get_cfl``, interp_vel's kinetic energy, ``cfg%integrate`` means
                                           -> nga_proj_flow_stats
* the channel's bulk velocities            -> nga_proj_bulk
* ``get_div`` and ``rhs = -vol*div*rho/dt`` -> nga_proj_divergence
* ``shift_p``                              -> nga_proj_shift_p
* ``get_pgrad``, ``P += sol``, ``U -= dt*grad/rho`` -> nga_proj_correct

Fields are CUDA float64 tensors in NGA2's padded layout [k, j, i] with
``ghost`` overlap layers; periodic overlaps hold the periodic images, walls
(non-periodic directions) keep the no-slip value 0 in their cells and faces.
There is no CPU path.
"""
from __future__ import annotations

import numpy as np

from . import bbmg as B
from .problems import STC7
from .projection import Projection

ALPHA = 0.7  # timetracker_class.f90:12, damping of dt increases


class TimeTracker:
    """NGA2's timetracker (src/libraries/timetracker_class.f90): dt from the
    CFL (``adjust_dt``, lines 88-97), time and step counters (``increment``,
    lines 68-84) and the sub-iteration counter."""

    def __init__(self, dtmax, cflmax, itmax=2, tmax=float("inf"), nmax=2 ** 62):
        self.dtmax, self.cflmax, self.itmax = float(dtmax), float(cflmax), int(itmax)
        self.tmax, self.nmax = tmax, nmax
        self.dt = self.dtmax
        self.dtold = self.dt
        self.cfl = 0.0
        self.t = 0.0
        self.n = 0
        self.it = 1

    def adjust_dt(self):
        self.dtold = self.dt
        if self.cfl > 0.0:
            self.dt = min(self.dtold * self.cflmax / self.cfl, self.dtmax)
        if self.dt > self.dtold:
            self.dt = ALPHA * self.dt + (1.0 - ALPHA) * self.dtold

    def increment(self):
        self.it = 1
        self.t = self.t + self.dt
        self.n += 1

    def done(self):
        return self.n >= self.nmax or self.t >= self.tmax


class Incomp:
    """The incompressible solver's state and operations on one triply
    periodic pgrid (node coordinates xn, yn, zn): U, V, W, P, Uold, Vold,
    Wold, the cell-centred viscosity, the constant density, and the pressure
    solver ``psolv`` set up once on ``-vol div(grad)`` (update_laplacian
    with rho = 1, incomp_class.f90:766-785)."""

    def __init__(self, xn, yn, zn, rho=1.0, visc=0.0, ghost=1, precision=B.FP64, rcvg=1e-10, maxit=100,
                 device=0, per=(True, True, True), implicit_rcvg=1e-6, implicit_maxit=100):
        import torch
        self.torch = torch
        self.per = tuple(bool(p) for p in per)
        self.proj = Projection(xn, yn, zn, *self.per, ghost=ghost, device=device)
        g = self.proj.grid
        self.nx, self.ny, self.nz, self.g = g.nx, g.ny, g.nz, ghost
        self.shape = self.proj.shape
        z = lambda: torch.zeros(self.shape, dtype=torch.float64, device="cuda")
        self.U, self.V, self.W, self.P = z(), z(), z(), z()
        self.Uold, self.Vold, self.Wold = z(), z(), z()
        self.resU, self.resV, self.resW = z(), z(), z()
        self.div, self.rhs, self.sol = z(), z(), z()
        self.rho = float(rho)
        self.visc = torch.full(self.shape, float(visc), dtype=torch.float64, device="cuda")
        self.rho_face = torch.full(self.shape, self.rho, dtype=torch.float64, device="cuda")
        self.opr = self.proj.update_laplacian()
        self.psolv = B.BBMG(self.nx, self.ny, self.nz, *self.per, ghost=ghost, method=B.PCG_BBOX,
                            precision=precision, rcvg=rcvg, maxit=maxit, device=device)
        self.psolv.setup(STC7, self.opr)
        self.psolv_it, self.psolv_rerr = 0, 0.0
        # the implicit velocity solver (created on first use): bbmg's multigrid
        # iteration, since the implicit operator is not symmetric
        self.implicit_rcvg, self.implicit_maxit, self.device = implicit_rcvg, implicit_maxit, device
        self.isolv = None
        self.implicit_its = []
        self.solve_ms = 0.0  # device time of the pressure solves, accumulated

    # ------------------------------------------------------------ operations
    def sync(self, a):
        """cfg%sync: the overlap of a padded field takes the periodic images
        (periodic directions only; the overlap of a wall direction is left)."""
        g = self.g
        if g == 0:
            return a
        for ax, per in ((2, self.per[0]), (1, self.per[1]), (0, self.per[2])):
            if not per:
                continue
            n = a.shape[ax] - 2 * g
            a.narrow(ax, 0, g).copy_(a.narrow(ax, n, g))
            a.narrow(ax, n + g, g).copy_(a.narrow(ax, g, g))
        return a

    def get_dmomdt(self):
        return self.proj.get_dmomdt(self.U, self.V, self.W, self.P, rho=self.rho, visc=self.visc,
                                    out=(self.resU, self.resV, self.resW))

    def get_div(self, dt=None):
        """div of the velocity; with dt also the pressure right-hand side
        rhs = -vol*div*rho/dt."""
        self.proj.get_div(self.U, self.V, self.W, rho=self.rho, dt=dt, div=self.div,
                          rhs=self.rhs if dt is not None else None)
        return self.div

    def stats(self, dt=1.0):
        return self.proj.flow_stats(self.U, self.V, self.W, visc=self.visc, rho=self.rho, dt=dt)

    def get_cfl(self, dt):
        """(cflc, cfl): the largest convective CFL and the largest overall."""
        s = self.stats(dt)
        cflc = max(s["cflc_x"], s["cflc_y"], s["cflc_z"])
        return cflc, max(cflc, s["cflv_x"], s["cflv_y"], s["cflv_z"])

    def solve_implicit(self, dt, res=None):
        """solve_implicit (incomp_class.f90:1744-1910): for U, V and W in
        turn, assemble the operator linearised about the current velocity,
        solve it from a zero guess with the component's residual as
        right-hand side, and replace the residual with the solution."""
        import torch
        res = res if res is not None else (self.resU, self.resV, self.resW)
        if self.isolv is None:
            self.isolv = B.BBMG(self.nx, self.ny, self.nz, *self.per, ghost=self.g, method=B.BBOX, precision=B.FP64,
                                rcvg=self.implicit_rcvg, maxit=self.implicit_maxit, device=self.device)
            self.iopr = torch.zeros(self.shape + (7,), dtype=torch.float64, device="cuda")
            self.isol = torch.zeros(self.shape, dtype=torch.float64, device="cuda")
        its = []
        for c, r in enumerate(res):
            self.proj.implicit_operator(c, dt, self.rho, self.U, self.V, self.W, visc=self.visc, opr=self.iopr)
            self.isolv.setup(STC7, self.iopr)
            self.isol.zero_()
            _, it, rerr, st = self.isolv.solve(r, self.isol)
            its.append(it)
            r.copy_(self.isol)
            self.sync(r)
        self.implicit_its.append(its)
        return its

    def pressure_projection(self, dt):
        """get_div, rhs = -vol*div*rho/dt, sol = 0, psolv%solve, shift_p,
        get_pgrad, P += sol, U -= dt*grad(sol)/rho (simulation.f90:332-343)."""
        self.get_div(dt)
        self.sol.zero_()
        _, it, rerr, st = self.psolv.solve(self.rhs, self.sol)
        self.psolv_it, self.psolv_rerr = it, rerr
        self.solve_ms += self.psolv.info["solve_ms"]
        self.proj.shift_p(self.sol)
        self.proj.correct(self.sol, dt, self.U, self.V, self.W, self.P, self.rho_face, self.rho_face, self.rho_face)
        return it, rerr, st

    def time_step(self, time, force=None, on_solve=None):
        """One step of the example's time loop (simulation.f90:262-352): dt
        from get_cfl and adjust_dt, Uold = U, then time.itmax sub-iterations
        of midpoint, get_dmomdt, explicit update and pressure projection.
        ``force(fs) -> (force_a, force_b, mean)`` supplies the linear forcing
        of each sub-iteration (None: unforced); ``on_solve(fs, prev_sol)`` is
        called after each pressure projection with the solution the solve
        replaced.  Returns each solve's PCG iteration count."""
        _, time.cfl = self.get_cfl(time.dt)
        time.adjust_dt()
        time.increment()
        for a, b in ((self.Uold, self.U), (self.Vold, self.V), (self.Wold, self.W)):
            a.copy_(b)
        its = []
        while time.it <= time.itmax:
            self.proj.midpoint(self.U, self.V, self.W, self.Uold, self.Vold, self.Wold)
            self.get_dmomdt()
            fa, fb, mean = force(self) if force is not None else (0.0, 1.0, None)
            self.proj.advance(time.dt, self.rho, self.U, self.V, self.W, self.Uold, self.Vold, self.Wold, self.resU,
                              self.resV, self.resW, force_a=fa, force_b=fb, mean=mean)
            prev = self.sol.clone() if on_solve is not None else None
            it, rerr, st = self.pressure_projection(time.dt)
            its.append(it)
            if on_solve is not None:
                on_solve(self, prev)
            time.it += 1
        self.get_div()
        return its

    def interior(self, a):
        g = self.g
        return a[g:g + self.nz, g:g + self.ny, g:g + self.nx]

    def close(self):
        if self.isolv is not None:
            self.isolv.close()
        self.psolv.close()
        self.proj.close()


class HIT:
    """The forced homogeneous isotropic turbulence example
    (examples/hit/src/simulation.f90) on the GPU: a (Lx)^3 triply periodic
    box of n^3 cells, Gaussian initial velocity of rms ``urms0`` projected to
    be divergence-free (lines 100-135), then the time loop (lines 256-352):
    dt from the CFL, ``itmax`` sub-iterations of a mid-point (Crank-Nicolson
    like) explicit update with linear forcing towards the initial kinetic
    energy, each closed by a pressure projection.  Defaults are the
    example's input file (examples/hit/input) without particles."""

    def __init__(self, n=64, Lx=1.0, visc=0.01, rho=1.0, urms0=5.0, tau_eddy=0.1, dtmax=1e-3, cflmax=0.9,
                 itmax=2, seed=0, ghost=1, precision=B.FP64, rcvg=1e-10, maxit=100, forcing=True, device=0):
        import torch
        self.torch = torch
        x = np.arange(n + 1, dtype=np.float64) / float(n) * Lx
        self.fs = Incomp(x, x, x, rho=rho, visc=visc, ghost=ghost, precision=precision, rcvg=rcvg, maxit=maxit,
                         device=device)
        self.time = TimeTracker(dtmax, cflmax, itmax)
        self.tau_eddy, self.forcing = float(tau_eddy), bool(forcing)
        self.records = []
        fs, g = self.fs, ghost
        rng = np.random.default_rng(seed)
        for a in (fs.U, fs.V, fs.W):  # random_normal(m=0, sd=Urms0) on the interior, then sync
            a[g:g + n, g:g + n, g:g + n] = torch.from_numpy(rng.normal(0.0, urms0, size=(n, n, n))).cuda()
            fs.sync(a)
        fs.pressure_projection(self.time.dt)
        self.KE0 = fs.stats()["KE"]
        self.KE = self.KE0

    def _force(self, fs):
        s = fs.stats()
        self.KE = s["KE"]
        return self.time.dt * self.KE0 / self.KE, 2.0 * self.tau_eddy, (s["meanU"], s["meanV"], s["meanW"])

    def step(self, keep=False):
        """One time step; returns the number of PCG iterations of each
        sub-iteration's pressure solve.  With keep, each solve's (rhs,
        previous solution, solution) is appended to ``records``."""
        keep_fn = (lambda fs, prev: self.records.append(self._record(prev))) if keep else None
        return self.fs.time_step(self.time, force=self._force if self.forcing else None, on_solve=keep_fn)

    def _record(self, prev):
        fs = self.fs
        inner = lambda a: fs.interior(a).contiguous()
        return {"rhs": inner(fs.rhs), "p_prev": inner(prev), "dp": inner(fs.sol), "dt": self.time.dt,
                "step": self.time.n, "it": fs.psolv_it}

    def close(self):
        self.fs.close()


def _face_mask(shape, g, ns, per, c):
    """umask (c = 0), vmask (1), wmask (2) > 0 on a padded array [k, j, i] for
    walls at both ends of every non-periodic direction (incomp_class.f90:
    196-242 with cfg%VF = 0 outside the domain)."""
    m = np.zeros(shape, bool)
    for d in range(3):
        if per[d]:
            continue
        idx = np.arange(-g, ns[d] + g)
        md = ((idx <= 0) | (idx >= ns[d])) if d == c else ((idx < 0) | (idx >= ns[d]))
        m |= md[None, None, :] if d == 0 else (md[None, :, None] if d == 1 else md[:, None, None])
    return m


def _centres(x, g):
    """Cell centres of the padded cells -g .. n+g-1 (the naive node extension)."""
    n = x.size - 1
    xe = np.empty(n + 1 + 2 * g)
    xe[g:g + n + 1] = x
    for m in range(g - 1, -1, -1):
        xe[m] = xe[m + 1] - (xe[g + 1] - xe[g])
    for m in range(g + n + 1, n + 1 + 2 * g):
        xe[m] = xe[m - 1] + (xe[g + n] - xe[g + n - 1])
    return 0.5 * (xe[:-1] + xe[1:])


class Channel:
    """The channel example (examples/channel/src/simulation.f90) on the GPU:
    x and z periodic, walls in y on the tanh-stretched grid of its
    geometry.f90 (lines 30-61), velocity initialised to the bulk values with
    the optional cosine perturbation (lines 147-167), then the time loop
    (lines 256-340): dt from the CFL, ``itmax`` sub-iterations of mid-point
    velocity, get_dmomdt, explicit residual with the bulk-velocity forcing of
    U and W, solve_implicit (three non-symmetric 7-point solves by bbmg
    multigrid), U = 2U - Uold + res and a pressure projection.  Defaults are
    the example's input file, with nz > 1 (the file's nz = 1 needs
    adjust_metrics' lower-dimension zeroing, which is not restated)."""

    def __init__(self, nx=128, ny=40, nz=8, Lx=5.0, Ly=1.0, Lz=0.04, stretch=2.1, visc=0.01, rho=1.0, Ubulk=1.0,
                 Wbulk=0.0, amp=0.0, dtmax=2e-2, cflmax=0.9, itmax=2, ghost=1, precision=B.FP64, rcvg=1e-10,
                 maxit=100, implicit_rcvg=1e-6, implicit_maxit=100, device=0):
        import torch
        x = np.arange(nx + 1, dtype=np.float64) / float(nx) * Lx
        j = np.arange(ny + 1, dtype=np.float64)
        y = 0.5 * Ly * np.tanh(stretch * (2.0 * j / float(ny) - 1.0)) / np.tanh(stretch)
        z = np.arange(nz + 1, dtype=np.float64) / float(nz) * Lz - 0.5 * Lz
        per = (True, False, True)
        self.fs = fs = Incomp(x, y, z, rho=rho, visc=visc, ghost=ghost, precision=precision, rcvg=rcvg, maxit=maxit,
                              device=device, per=per, implicit_rcvg=implicit_rcvg, implicit_maxit=implicit_maxit)
        self.time = TimeTracker(dtmax, cflmax, itmax)
        self.Ubulk, self.Wbulk = float(Ubulk), float(Wbulk)
        g, ns = ghost, (nx, ny, nz)
        vel = np.sqrt(Ubulk ** 2 + Wbulk ** 2)
        zm = _centres(z, g)[:, None, None]
        xm = _centres(x, g)[None, None, :]
        one = np.ones(fs.shape)
        um, wm = _face_mask(fs.shape, g, ns, per, 0), _face_mask(fs.shape, g, ns, per, 2)
        U = np.where(um, 0.0, Ubulk * one)
        U = np.where(um, U, U + amp * vel * np.cos(8.0 * 2.0 * np.pi * zm / Lz))
        W = np.where(wm, 0.0, Wbulk * one)
        W = np.where(wm, W, W + amp * vel * np.cos(8.0 * 2.0 * np.pi * xm / Lx))
        fs.U.copy_(torch.from_numpy(U))
        fs.W.copy_(torch.from_numpy(W))
        self.meanU, self.meanW = self.Ubulk, self.Wbulk

    def step(self):
        """One time step; returns the pressure solves' PCG iterations."""
        fs, time = self.fs, self.time
        _, time.cfl = fs.get_cfl(time.dt)
        time.adjust_dt()
        time.increment()
        for a, b in ((fs.Uold, fs.U), (fs.Vold, fs.V), (fs.Wold, fs.W)):
            a.copy_(b)
        its = []
        while time.it <= time.itmax:
            fs.proj.midpoint(fs.U, fs.V, fs.W, fs.Uold, fs.Vold, fs.Wold)
            fs.get_dmomdt()
            (su, vu), _, (sw, vw) = fs.proj.bulk(fs.U, fs.V, fs.W, fs.Uold, fs.Vold, fs.Wold)
            self.meanU, self.meanW = su / vu, sw / vw
            fs.proj.mom_residual(time.dt, fs.rho, fs.U, fs.V, fs.W, fs.Uold, fs.Vold, fs.Wold, fs.resU, fs.resV,
                                 fs.resW, force={0: (self.Ubulk, self.meanU), 2: (self.Wbulk, self.meanW)})
            fs.solve_implicit(time.dt)
            fs.proj.apply_residual(fs.U, fs.V, fs.W, fs.Uold, fs.Vold, fs.Wold, fs.resU, fs.resV, fs.resW)
            it, rerr, st = fs.pressure_projection(time.dt)
            its.append(it)
            time.it += 1
        fs.get_div()
        return its

    def close(self):
        self.fs.close()
