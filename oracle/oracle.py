"""ctypes front end of the CPU oracle (bbmg_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline legs, to check the GPU solver; the product never imports it.

``OracleBBMG`` mirrors NGA2's ILS bbmg branch (src/solver/ils_class.f90:162-226
init, 230-376 setup, 674-822 solve): methods ``bbox`` (stationary V-cycles) and
``pcg_bbox`` (V-cycle preconditioned CG) with V(2,2), a direct coarsest solve and
``ncell_coarsest = 300``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

BBOX, PCG_BBOX = 1, 2
WHICH = {"opr": 0, "c2f": 1, "f2c": 2, "oprc2f": 3, "v": 4, "f": 5, "r": 6}
NCOEF = {"opr": 27, "c2f": 8, "f2c": 27, "oprc2f": 27, "v": 1, "f": 1, "r": 1}


def build(release: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc only) and return the .so path."""
    name = "liboracle_bbmg_release.so" if release else "liboracle_bbmg.so"
    path = os.path.join(HERE, name)
    src = os.path.join(HERE, "bbmg_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, path], check=True)
    return path


def load(release: bool = False):
    key = bool(release)
    if key in _LIBS:
        return _LIBS[key]
    lib = C.CDLL(build(release))
    P, I, D = C.c_void_p, C.c_int, C.c_double
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    lib.orc_create.restype = P
    lib.orc_create.argtypes = [I, I, I, I, I, I, I, D, I, I, I, I, I, I]
    lib.orc_destroy.argtypes = [P]
    lib.orc_nlvl.restype = I
    lib.orc_nlvl.argtypes = [P]
    lib.orc_level_dims.argtypes = [P, I, ip]
    lib.orc_set_operator.argtypes = [P, I, ip, dp, I]
    lib.orc_update.argtypes = [P]
    for f in ("orc_recompute_prolongation", "orc_recompute_restriction", "orc_recompute_operator",
              "orc_get_residual", "orc_f2c", "orc_c2f", "orc_cycle"):
        getattr(lib, f).argtypes = [P, I]
    lib.orc_recompute_direct.argtypes = [P]
    lib.orc_relax.argtypes = [P, I, I]
    lib.orc_direct_solve.argtypes = [P]
    lib.orc_bbmg_solve.argtypes = [P]
    lib.orc_solve.argtypes = [P, dp, dp, ip, dp]
    lib.orc_get.restype = C.c_long
    lib.orc_get.argtypes = [P, I, I, dp]
    lib.orc_put.restype = C.c_long
    lib.orc_put.argtypes = [P, I, I, dp]
    lib.orc_direct_info.restype = I
    lib.orc_direct_info.argtypes = [P, ip]
    lib.orc_get_direct.restype = C.c_long
    lib.orc_get_direct.argtypes = [P, dp, dp, ip]
    lib.orc_direct_apply.argtypes = [P, dp]
    lib.orc_set_params.argtypes = [P, I, D]
    lib.orc_set_pin_singular.argtypes = [P, I]
    lib.orc_npinned.restype = I
    lib.orc_npinned.argtypes = [P]
    _LIBS[key] = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class OracleBBMG:
    """One bbmg instance on one rank (the ILS-driven configuration)."""

    def __init__(self, nx, ny, nz, xper, yper, zper, method=PCG_BBOX, maxit=100, rcvg=1e-10,
                 relax_pre=2, relax_post=2, ncell_coarsest=300, use_direct_solve=True, ncycle=1,
                 release=False, pin_singular=True):
        self.lib = load(release)
        self.shape = (nz, ny, nx)
        self.per = (bool(xper), bool(yper), bool(zper))
        self.method = method
        self.h = self.lib.orc_create(nx, ny, nz, int(xper), int(yper), int(zper), maxit, rcvg, ncycle,
                                     relax_pre, relax_post, ncell_coarsest, int(use_direct_solve),
                                     int(method == PCG_BBOX))
        if not self.h:
            raise MemoryError("oracle allocation failed")
        self.lib.orc_set_pin_singular(self.h, int(pin_singular))

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nlvl(self):
        return self.lib.orc_nlvl(self.h)

    def level_dims(self, n):
        d = np.zeros(3, np.int32)
        self.lib.orc_level_dims(self.h, n, _ip(d))
        return tuple(int(x) for x in d)

    def set_params(self, maxit, rcvg):
        self.lib.orc_set_params(self.h, maxit, rcvg)

    # -- setup ------------------------------------------------------------
    def set_operator(self, stc, opr, ghost=0):
        """``opr`` is (nz+2g, ny+2g, nx+2g, nst) (Fortran opr(st,i,j,k))."""
        stc = np.ascontiguousarray(stc, np.int32)
        opr = np.ascontiguousarray(opr, np.float64)
        self.lib.orc_set_operator(self.h, stc.shape[0], _ip(stc), _dp(opr), ghost)

    def update(self):
        self.lib.orc_update(self.h)

    def setup(self, stc, opr, ghost=0):
        self.set_operator(stc, opr, ghost)
        self.update()

    # -- solve ------------------------------------------------------------
    def solve(self, rhs, sol=None):
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.zeros(self.shape) if sol is None else np.array(sol, np.float64, order="C", copy=True)
        it = C.c_int(0)
        rerr = C.c_double(0.0)
        self.lib.orc_solve(self.h, _dp(rhs), _dp(x), C.byref(it), C.byref(rerr))
        return x, it.value, rerr.value

    # -- per-step access for parity tests ----------------------------------
    def get(self, n, which):
        nz, ny, nx = [d + 2 for d in reversed(self.level_dims(n))]
        cnt = self.lib.orc_get(self.h, n, WHICH[which], None)
        if cnt < 0:
            raise KeyError(f"{which} absent on level {n}")
        out = np.empty(cnt)
        self.lib.orc_get(self.h, n, WHICH[which], _dp(out))
        nc = NCOEF[which]
        return out.reshape((nz, ny, nx, nc) if nc > 1 else (nz, ny, nx))

    def put(self, n, which, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        if self.lib.orc_put(self.h, n, WHICH[which], _dp(arr)) < 0:
            raise KeyError(f"{which} absent on level {n}")

    def relax(self, n, direction):
        self.lib.orc_relax(self.h, n, direction)

    def residual(self, n):
        self.lib.orc_get_residual(self.h, n)

    def restrict(self, nf):
        self.lib.orc_f2c(self.h, nf)

    def prolong(self, nc):
        self.lib.orc_c2f(self.h, nc)

    def cycle(self, n=1):
        self.lib.orc_cycle(self.h, n)

    def direct_solve(self):
        self.lib.orc_direct_solve(self.h)

    def bbmg_solve(self):
        self.lib.orc_bbmg_solve(self.h)

    def recompute_prolongation(self, n):
        self.lib.orc_recompute_prolongation(self.h, n)

    def recompute_restriction(self, n):
        self.lib.orc_recompute_restriction(self.h, n)

    def recompute_operator(self, n):
        self.lib.orc_recompute_operator(self.h, n)

    def recompute_direct(self):
        self.lib.orc_recompute_direct(self.h)

    def direct(self):
        np_ = C.c_int(0)
        info = self.lib.orc_direct_info(self.h, C.byref(np_))
        n = np_.value
        OP = np.empty(n * n); LU = np.empty(n * n); piv = np.empty(n, np.int32)
        self.lib.orc_get_direct(self.h, _dp(OP), _dp(LU), _ip(piv))
        # column-major (Fortran) -> row-major matrix
        return OP.reshape(n, n).T.copy(), LU.reshape(n, n).T.copy(), piv, info

    @property
    def npinned(self):
        return self.lib.orc_npinned(self.h)

    def direct_apply(self, b):
        x = np.array(b, np.float64, copy=True)
        self.lib.orc_direct_apply(self.h, _dp(x))
        return x


def fft_solve_periodic(opr7, rhs):
    """Exact solution of a triply periodic constant-coefficient 7-point system.

    The operator is circulant, so it is diagonal in the discrete Fourier basis
    (the method of src/solver/fourier3d_class.f90:1128-1202); the zero mode is
    set to zero, i.e. the solution has zero mean."""
    a = opr7[0, 0, 0]
    nz, ny, nx = rhs.shape
    kx = np.exp(2j * np.pi * np.fft.fftfreq(nx))
    ky = np.exp(2j * np.pi * np.fft.fftfreq(ny))
    kz = np.exp(2j * np.pi * np.fft.fftfreq(nz))
    lam = (a[0] + a[1] * kx[None, None, :] + a[2] / kx[None, None, :]
           + a[3] * ky[None, :, None] + a[4] / ky[None, :, None]
           + a[5] * kz[:, None, None] + a[6] / kz[:, None, None])
    rh = np.fft.fftn(rhs)
    lam[0, 0, 0] = 1.0
    ph = rh / lam
    ph[0, 0, 0] = 0.0
    return np.fft.ifftn(ph).real
