"""Python side of the GPU projection steps (include/nga_projection.h).

The names follow NGA2's flow solvers: ``update_laplacian``, ``get_div``,
``shift_p``, ``get_pgrad``, plus ``correct`` for the velocity correction of the
time loop.  Arrays are CUDA float64 torch tensors in NGA2's padded layout
[k, j, i] (shape (nz+2g, ny+2g, nx+2g)); the operator is [k, j, i, 7].  There
is no CPU path: the library must be built and a GPU present.
"""
from __future__ import annotations

import ctypes as C

from . import bbmg as B

EXPORTS = ["nga_proj_create", "nga_proj_destroy", "nga_proj_set_stream", "nga_proj_laplacian",
           "nga_proj_divergence", "nga_proj_shift_p", "nga_proj_pgrad", "nga_proj_correct", "nga_proj_dmomdt",
           "nga_proj_midpoint", "nga_proj_advance", "nga_proj_flow_stats", "nga_proj_implicit_operator",
           "nga_proj_mom_residual", "nga_proj_apply_residual", "nga_proj_bulk"]

_BOUND = False


def lib():
    global _BOUND
    L = B.load()
    if not _BOUND:
        P, I, D = C.c_void_p, C.c_int, C.c_double
        DP = C.POINTER(C.c_double)
        L.nga_proj_create.argtypes = [C.POINTER(B.Grid), DP, DP, DP, I, C.POINTER(P)]
        L.nga_proj_destroy.argtypes = [P]
        L.nga_proj_set_stream.argtypes = [P, P]
        L.nga_proj_laplacian.argtypes = [P, P, P, P, P]
        L.nga_proj_divergence.argtypes = [P, P, P, P, D, D, P, P]
        L.nga_proj_shift_p.argtypes = [P, P, DP]
        L.nga_proj_pgrad.argtypes = [P, P, P, P, P]
        L.nga_proj_correct.argtypes = [P, P, D, P, P, P, P, P, P, P]
        L.nga_proj_dmomdt.argtypes = [P, P, P, P, P, D, P, D, P, P, P]
        L.nga_proj_midpoint.argtypes = [P, P, P, P, P, P, P]
        L.nga_proj_advance.argtypes = [P, D, D, P, P, P, P, P, P, P, P, P, D, D, DP]
        L.nga_proj_flow_stats.argtypes = [P, P, P, P, P, D, D, D, DP]
        L.nga_proj_implicit_operator.argtypes = [P, I, D, D, P, P, P, P, D, P]
        L.nga_proj_mom_residual.argtypes = [P, D, D, P, P, P, P, P, P, P, P, P, I, DP]
        L.nga_proj_apply_residual.argtypes = [P, P, P, P, P, P, P, P, P, P]
        L.nga_proj_bulk.argtypes = [P, P, P, P, P, P, P, DP]
        for n in EXPORTS:
            getattr(L, n).restype = C.c_int
        _BOUND = True
    return L


def _p(t):
    if t is None:
        return None
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise TypeError("projection arrays must be contiguous CUDA float64 tensors")
    return t.data_ptr()


class Projection:
    """The projection steps of one pgrid (node coordinates xn, yn, zn)."""

    def __init__(self, xn, yn, zn, xper, yper, zper, ghost=1, device=-1):
        import numpy as np
        self.lib = lib()
        xn, yn, zn = (np.ascontiguousarray(a, dtype=np.float64) for a in (xn, yn, zn))
        self.grid = B.Grid(xn.size - 1, yn.size - 1, zn.size - 1, int(xper), int(yper), int(zper), ghost)
        self.h = C.c_void_p()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.nga_proj_create(C.byref(self.grid), dp(xn), dp(yn), dp(zn), device, C.byref(self.h)))
        self.shape = (self.grid.nz + 2 * ghost, self.grid.ny + 2 * ghost, self.grid.nx + 2 * ghost)

    def _check(self, st):
        if st != 0:
            msg = self.lib.bbmg_last_error(None)
            raise RuntimeError(f"projection status {st}: {msg.decode() if msg else ''}")

    def _new(self, *extra):
        import torch
        return torch.zeros(self.shape + tuple(extra), dtype=torch.float64, device="cuda")

    def set_stream(self, stream):
        self._check(self.lib.nga_proj_set_stream(self.h, stream))

    def update_laplacian(self, rho_U=None, rho_V=None, rho_W=None, opr=None):
        opr = self._new(7) if opr is None else opr
        self._check(self.lib.nga_proj_laplacian(self.h, _p(rho_U), _p(rho_V), _p(rho_W), _p(opr)))
        return opr

    def get_div(self, U, V, W, rho=1.0, dt=None, div=None, rhs=None, want_div=True):
        if want_div and div is None:
            div = self._new()
        if dt is not None and rhs is None:
            rhs = self._new()
        self._check(self.lib.nga_proj_divergence(self.h, _p(U), _p(V), _p(W), float(rho),
                                                 float(dt if dt is not None else 0.0), _p(div), _p(rhs)))
        return div, rhs

    def shift_p(self, pressure):
        m = C.c_double(0.0)
        self._check(self.lib.nga_proj_shift_p(self.h, _p(pressure), C.byref(m)))
        return m.value

    def get_pgrad(self, P, gx=None, gy=None, gz=None):
        gx = self._new() if gx is None else gx
        gy = self._new() if gy is None else gy
        gz = self._new() if gz is None else gz
        self._check(self.lib.nga_proj_pgrad(self.h, _p(P), _p(gx), _p(gy), _p(gz)))
        return gx, gy, gz

    def correct(self, sol, dt, U, V, W, P=None, rho_U=None, rho_V=None, rho_W=None):
        self._check(self.lib.nga_proj_correct(self.h, _p(sol), float(dt), _p(rho_U), _p(rho_V), _p(rho_W),
                                              _p(P), _p(U), _p(V), _p(W)))

    def get_dmomdt(self, U, V, W, P, rho=1.0, visc=None, visc0=0.0, out=None):
        """Time derivatives of rho U, rho V, rho W (incomp's get_dmomdt); a
        non-periodic direction has walls at both ends; visc is a cell-centred
        array or None for visc0."""
        dU, dV, dW = out if out is not None else (self._new(), self._new(), self._new())
        self._check(self.lib.nga_proj_dmomdt(self.h, _p(U), _p(V), _p(W), _p(P), float(rho), _p(visc), float(visc0),
                                             _p(dU), _p(dV), _p(dW)))
        return dU, dV, dW

    def midpoint(self, U, V, W, Uold, Vold, Wold):
        """U = 0.5*(U + Uold), V and W likewise, in place."""
        self._check(self.lib.nga_proj_midpoint(self.h, _p(U), _p(V), _p(W), _p(Uold), _p(Vold), _p(Wold)))

    def advance(self, dt, rho, U, V, W, Uold, Vold, Wold, dU, dV, dW, force_a=0.0, force_b=1.0, mean=None):
        """The explicit update of a sub-iteration, in place on U, V, W:
        U = 2U - Uold + (-2(rho U - rho Uold) + dt dU [+ (force_a (U - mean))/force_b])/rho."""
        m = (C.c_double * 3)(*(mean if mean is not None else (0.0, 0.0, 0.0)))
        self._check(self.lib.nga_proj_advance(self.h, float(dt), float(rho), _p(U), _p(V), _p(W), _p(Uold), _p(Vold),
                                              _p(Wold), _p(dU), _p(dV), _p(dW), float(force_a), float(force_b), m))

    def flow_stats(self, U, V, W, visc=None, visc0=0.0, rho=1.0, dt=1.0):
        """dict of get_cfl's CFLs (cflc_x/y/z, cflv_x/y/z), the kinetic energy KE
        of the cell-interpolated velocity and the mean velocities meanU/V/W."""
        out = (C.c_double * 10)()
        self._check(self.lib.nga_proj_flow_stats(self.h, _p(U), _p(V), _p(W), _p(visc), float(visc0), float(rho),
                                                 float(dt), out))
        keys = ("cflc_x", "cflc_y", "cflc_z", "cflv_x", "cflv_y", "cflv_z", "KE", "meanU", "meanV", "meanW")
        return dict(zip(keys, list(out)))

    def implicit_operator(self, comp, dt, rho, U, V, W, visc=None, visc0=0.0, opr=None):
        """solve_implicit's 7-point operator for component comp (0 U, 1 V, 2 W)."""
        opr = self._new(7) if opr is None else opr
        self._check(self.lib.nga_proj_implicit_operator(self.h, int(comp), float(dt), float(rho), _p(U), _p(V),
                                                        _p(W), _p(visc), float(visc0), _p(opr)))
        return opr

    def mom_residual(self, dt, rho, U, V, W, Uold, Vold, Wold, resU, resV, resW, force=None):
        """res = -2(rho U - rho Uold) + dt res in place; force maps a component
        (0, 1, 2) to (a, b): res = (res + a) - b on its unmasked faces."""
        f = (C.c_double * 6)()
        mask = 0
        for c, (a, b) in (force or {}).items():
            f[2 * c], f[2 * c + 1] = float(a), float(b)
            mask |= 1 << c
        self._check(self.lib.nga_proj_mom_residual(self.h, float(dt), float(rho), _p(U), _p(V), _p(W), _p(Uold),
                                                   _p(Vold), _p(Wold), _p(resU), _p(resV), _p(resW), mask, f))

    def apply_residual(self, U, V, W, Uold, Vold, Wold, resU, resV, resW):
        """U = 2U - Uold + resU, V and W likewise, in place."""
        self._check(self.lib.nga_proj_apply_residual(self.h, _p(U), _p(V), _p(W), _p(Uold), _p(Vold), _p(Wold),
                                                     _p(resU), _p(resV), _p(resW)))

    def bulk(self, U, V, W, Uold, Vold, Wold):
        """[(sum w (2U - Uold), sum w) for U, V, W] over the unmasked faces."""
        out = (C.c_double * 6)()
        self._check(self.lib.nga_proj_bulk(self.h, _p(U), _p(V), _p(W), _p(Uold), _p(Vold), _p(Wold), out))
        return [(out[2 * c], out[2 * c + 1]) for c in range(3)]

    def close(self):
        if self.h:
            self.lib.nga_proj_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
