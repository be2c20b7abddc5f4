"""Python front end of the B200 bbmg pressure solver (ctypes over libbbmg_b200.so).

Two layers:

* ``BBMG`` -- one-to-one with the C ABI in ``include/bbmg_b200.h``.
* ``ILS``  -- the linear-solver interface NGA2's flow solvers program against
  (``src/solver/linsol_class.f90:16-58``, ``src/solver/ils_class.f90:48-105``):
  public ``stc``, ``opr``, ``rhs``, ``sol``, ``maxit``, ``rcvg``, ``it``,
  ``rerr`` and the calls ``init()``, ``setup()``, ``solve()``, ``destroy()``.

Arrays are NGA2's: ``opr[k, j, i, st]`` (``opr(st,i,j,k)``), vectors ``[k, j, i]``,
each direction padded by ``ghost`` overlap layers.  numpy arrays are host memory;
torch CUDA tensors are passed as device pointers.  There is no CPU fallback:
without the library or a GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbbmg_b200.so")

BBOX, PCG_BBOX = 1, 2
FP64, MIXED = 0, 1
NORM_GUESS, NORM_RHS = 0, 1
STATUS = {0: "OK", 1: "MAXIT", 2: "STAGNATION", 3: "NONFINITE", 4: "BAD_ARGS", 5: "NOT_SETUP",
          6: "CUDA", 7: "NO_MEMORY"}
ARR = {"opr": 0, "c2f": 1, "f2c": 2, "oprc2f": 3, "v": 4, "f": 5, "r": 6}
STEP = {"relax": 0, "residual": 1, "restrict": 2, "prolong": 3, "cycle": 4, "direct": 5}
EXPORTS = ["bbmg_default_params", "bbmg_create", "bbmg_setup", "bbmg_solve", "bbmg_set_convergence",
           "bbmg_set_residual_norm",
           "bbmg_set_stream", "bbmg_get_info", "bbmg_destroy", "bbmg_last_error", "bbmg_debug_get",
           "bbmg_debug_put", "bbmg_debug_step", "bbmg_debug_direct", "bbmg_profile_step",
           "bbmg_residual_norm_noalloc", "bbmg_set_precond_stage"]


class BBMGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"bbmg status {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("xper", C.c_int), ("yper", C.c_int),
                ("zper", C.c_int), ("ghost", C.c_int)]


class Params(C.Structure):
    _fields_ = [("method", C.c_int), ("precision", C.c_int), ("ncycle", C.c_int), ("relax_pre", C.c_int),
                ("relax_post", C.c_int), ("ncell_coarsest", C.c_int), ("use_direct_solve", C.c_int),
                ("maxit", C.c_int), ("rcvg", C.c_double), ("device", C.c_int)]


class Info(C.Structure):
    _fields_ = [("nlvl", C.c_int), ("level_dims", (C.c_int * 3) * 16), ("coarse_n", C.c_int),
                ("coarse_pinned", C.c_int), ("it", C.c_int), ("rerr", C.c_double), ("res0", C.c_double),
                ("true_rerr", C.c_double), ("setup_ms", C.c_double), ("solve_ms", C.c_double),
                ("device_bytes", C.c_longlong), ("status", C.c_int), ("launches", C.c_longlong),
                ("level1_stencil", C.c_int), ("fallback_it", C.c_int), ("true_res", C.c_double),
                ("l2_rerr", C.c_double), ("stage_it", C.c_int)]


# first preconditioner stage: int fn(void *ctx, const double *r, double *z, void *stream)
STAGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)


_LIB = None


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `python -m nga2_b200.build`")
    lib = C.CDLL(path)
    P, I, D = C.c_void_p, C.c_int, C.c_double
    lib.bbmg_default_params.argtypes = [C.POINTER(Params)]
    lib.bbmg_default_params.restype = None
    lib.bbmg_create.argtypes = [C.POINTER(Grid), C.POINTER(Params), C.POINTER(P)]
    lib.bbmg_setup.argtypes = [P, I, C.POINTER(C.c_int), P]
    lib.bbmg_solve.argtypes = [P, P, P, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.bbmg_set_convergence.argtypes = [P, I, D]
    lib.bbmg_set_residual_norm.argtypes = [P, I]
    lib.bbmg_set_stream.argtypes = [P, P]
    lib.bbmg_get_info.argtypes = [P, C.POINTER(Info)]
    lib.bbmg_destroy.argtypes = [P]
    lib.bbmg_last_error.argtypes = [P]
    lib.bbmg_last_error.restype = C.c_char_p
    lib.bbmg_debug_get.argtypes = [P, I, I, I, P]
    lib.bbmg_debug_get.restype = C.c_longlong
    lib.bbmg_debug_put.argtypes = [P, I, I, I, P]
    lib.bbmg_debug_put.restype = C.c_longlong
    lib.bbmg_debug_step.argtypes = [P, I, I, I, I]
    lib.bbmg_debug_direct.argtypes = [P, P, P, P, C.POINTER(C.c_int)]
    lib.bbmg_profile_step.argtypes = [P, I, I, I, I, I, C.POINTER(C.c_double)]
    lib.bbmg_set_precond_stage.argtypes = [P, STAGE_FN, P, I, P, P]
    _LIB = lib
    return lib


def default_params() -> Params:
    p = Params()
    load().bbmg_default_params(C.byref(p))
    return p


def _ptr(a):
    """(pointer, keepalive) for a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("arrays must be C-contiguous float64")
        return a.ctypes.data, a
    if hasattr(a, "data_ptr"):
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("tensors must be contiguous float64")
        return a.data_ptr(), a
    raise TypeError(f"unsupported array type {type(a)}")


class BBMG:
    """One solver handle (the C ABI's bbmg_handle)."""

    def __init__(self, nx, ny, nz, xper, yper, zper, ghost=0, method=PCG_BBOX, precision=FP64, maxit=100,
                 rcvg=1e-10, relax_pre=2, relax_post=2, ncell_coarsest=300, use_direct_solve=True, ncycle=1,
                 device=-1):
        self.lib = load()
        self.grid = Grid(nx, ny, nz, int(xper), int(yper), int(zper), ghost)
        self.params = default_params()
        self.params.method = method
        self.params.precision = precision
        self.params.maxit = maxit
        self.params.rcvg = rcvg
        self.params.relax_pre = relax_pre
        self.params.relax_post = relax_post
        self.params.ncell_coarsest = ncell_coarsest
        self.params.use_direct_solve = int(use_direct_solve)
        self.params.ncycle = ncycle
        self.params.device = device
        self.h = C.c_void_p()
        st = self.lib.bbmg_create(C.byref(self.grid), C.byref(self.params), C.byref(self.h))
        if st:
            raise BBMGError(st, self.lib.bbmg_last_error(None).decode())
        self.shape = (nz + 2 * ghost, ny + 2 * ghost, nx + 2 * ghost)

    # ---------------------------------------------------------------- helpers
    def _check(self, st, allow=(0,)):
        if st not in allow:
            raise BBMGError(st, self.lib.bbmg_last_error(self.h).decode())
        return st

    def close(self):
        if self.h:
            self.lib.bbmg_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------- API
    def setup(self, stc, opr):
        stc = np.ascontiguousarray(stc, np.int32)
        p, keep = _ptr(opr)
        self._check(self.lib.bbmg_setup(self.h, stc.shape[0], stc.ctypes.data_as(C.POINTER(C.c_int)), p))

    def solve(self, rhs, sol=None, allow=(0, 1, 2)):
        """Solve in place into ``sol`` (a fresh zero guess if None).
        Returns ``(sol, it, rerr, status)``; statuses not in ``allow`` raise."""
        if sol is None:
            sol = np.zeros(self.shape) if isinstance(rhs, np.ndarray) else rhs.new_zeros(rhs.shape)
        pr, k1 = _ptr(rhs)
        ps, k2 = _ptr(sol)
        it = C.c_int(0)
        rerr = C.c_double(0.0)
        st = self.lib.bbmg_solve(self.h, pr, ps, C.byref(it), C.byref(rerr))
        self._check(st, allow)
        return sol, it.value, rerr.value, st

    def set_convergence(self, maxit, rcvg):
        self._check(self.lib.bbmg_set_convergence(self.h, maxit, rcvg))

    def set_residual_norm(self, norm):
        """NORM_GUESS (the reference's rerr) or NORM_RHS (rerr = max|r| / max|rhs|)."""
        self._check(self.lib.bbmg_set_residual_norm(self.h, norm))

    def set_precond_stage(self, fn, r=None, z=None, iters=0):
        """First preconditioner stage for mixed pcg_bbox (``fn`` None removes it).
        ``r`` and ``z`` are contiguous float64 CUDA tensors of shape (nz, ny, nx)
        (no overlap): before each call ``fn(r, z, stream_ptr)`` the solver
        writes the residual into ``r``; ``fn`` writes its approximation of
        A^-1 r into ``z``, enqueuing its work on the CUDA stream ``stream_ptr``.
        An exception in ``fn`` ends the solve with BAD_ARGS (kept in
        ``stage_error``).  ``iters``: leading iterations that apply it (0 = all)."""
        if fn is None:
            self._stage = None
            self._check(self.lib.bbmg_set_precond_stage(self.h, STAGE_FN(), None, 0, None, None))
            return
        want = self.shape if self.grid.ghost == 0 else (self.grid.nz, self.grid.ny, self.grid.nx)
        for t in (r, z):
            if tuple(t.shape) != tuple(want):
                raise ValueError(f"stage arrays must have shape {want}")
        pr, _ = _ptr(r)
        pz, _ = _ptr(z)

        def call(ctx, rp, zp, stream):
            try:
                fn(r, z, stream)
                return 0
            except Exception as e:  # noqa: BLE001 -- reported through the status
                self.stage_error = e
                return 1
        self.stage_error = None
        self._stage = (STAGE_FN(call), r, z)  # kept alive with the handle
        self._check(self.lib.bbmg_set_precond_stage(self.h, self._stage[0], None, iters, pr, pz))

    def set_stream(self, stream_ptr):
        self._check(self.lib.bbmg_set_stream(self.h, C.c_void_p(stream_ptr)))

    @property
    def info(self) -> dict:
        inf = Info()
        self._check(self.lib.bbmg_get_info(self.h, C.byref(inf)))
        d = {k: getattr(inf, k) for k, _ in Info._fields_ if k != "level_dims"}
        d["level_dims"] = [tuple(inf.level_dims[n]) for n in range(inf.nlvl)]
        return d

    @property
    def nlvl(self):
        return self.info["nlvl"]

    def level_dims(self, n):
        return self.info["level_dims"][n - 1]

    # ------------------------------------------------------ step-level access
    def get(self, n, which, prec=0):
        cnt = self.lib.bbmg_debug_get(self.h, n, ARR[which], prec, None)
        if cnt < 0:
            self._check(-cnt)
        out = np.empty(cnt)
        self.lib.bbmg_debug_get(self.h, n, ARR[which], prec, out.ctypes.data)
        nx, ny, nz = self.level_dims(n)
        nc = cnt // ((nx + 2) * (ny + 2) * (nz + 2))
        return out.reshape((nz + 2, ny + 2, nx + 2, nc) if nc > 1 else (nz + 2, ny + 2, nx + 2))

    def put(self, n, which, arr, prec=0):
        arr = np.ascontiguousarray(arr, np.float64)
        r = self.lib.bbmg_debug_put(self.h, n, ARR[which], prec, arr.ctypes.data)
        if r < 0:
            self._check(-r)

    def step(self, name, n, arg=0, prec=0):
        self._check(self.lib.bbmg_debug_step(self.h, STEP[name], n, arg, prec))

    def profile(self, name, n, arg=0, prec=0, reps=20):
        """Average device milliseconds of one stage (run `reps` times back to back)."""
        ms = C.c_double(0.0)
        self._check(self.lib.bbmg_profile_step(self.h, STEP[name], n, arg, prec, reps, C.byref(ms)))
        return ms.value

    def direct(self):
        npv = C.c_int(0)
        self.lib.bbmg_debug_direct(self.h, None, None, None, C.byref(npv))
        n = npv.value
        op = np.empty((n, n)); lu = np.empty((n, n)); piv = np.empty(n, np.int32)
        self._check(self.lib.bbmg_debug_direct(self.h, op.ctypes.data, lu.ctypes.data, piv.ctypes.data,
                                               C.byref(npv)))
        return op, lu, piv


class ILS:
    """NGA2's linear-solver object for the bbmg methods, on the GPU.

    Usage mirrors the Fortran (``ils_class.f90``)::

        ps = ILS(nx, ny, nz, xper, yper, zper, ghost=no, nst=7, maxit=100, rcvg=1e-10)
        ps.stc[:] = STC7; ps.opr[...] = ...       # caller-assembled operator
        ps.init(PCG_BBOX); ps.setup()
        ps.rhs[...] = ...; ps.sol[...] = 0.0; ps.solve(); print(ps.it, ps.rerr)
    """

    def __init__(self, nx, ny, nz, xper, yper, zper, ghost=0, nst=7, maxit=100, rcvg=1e-10,
                 precision=FP64, name="pressure"):
        self.name = name
        self.dims = (nx, ny, nz)
        self.per = (xper, yper, zper)
        self.ghost = ghost
        self.nst = nst
        shape = (nz + 2 * ghost, ny + 2 * ghost, nx + 2 * ghost)
        self.stc = np.zeros((nst, 3), np.int32)
        self.opr = np.zeros(shape + (nst,))
        self.rhs = np.zeros(shape)
        self.sol = np.zeros(shape)
        self.maxit = maxit
        self.rcvg = rcvg
        self.acvg = 0.0
        self.it = -1
        self.rerr = float("inf")
        self.aerr = float("inf")
        self.precision = precision
        self.method = None
        self.setup_done = False
        self._h = None

    def init(self, method):
        """ils%init: build the hierarchy (ils_class.f90:162-226)."""
        if method not in (BBOX, PCG_BBOX):
            raise ValueError("[ils init] Unknown solution method")
        self.method = method
        nx, ny, nz = self.dims
        self._h = BBMG(nx, ny, nz, *self.per, ghost=self.ghost, method=method, precision=self.precision,
                       maxit=self.maxit, rcvg=self.rcvg)

    def setup(self):
        """ils%setup: copy the operator and rebuild the levels (ils_class.f90:230-376)."""
        if self._h is None:
            raise RuntimeError("[ils setup] init has not been called")
        self._h.setup(self.stc, self.opr)
        self.setup_done = True

    def solve(self):
        """ils%solve: it/rerr as the reference reports them (ils_class.f90:674-822)."""
        if not self.setup_done:
            raise RuntimeError("[ils solve] Solver has not been setup.")
        self._h.set_convergence(self.maxit, self.rcvg)
        _, self.it, self.rerr, _ = self._h.solve(self.rhs, self.sol)

    def destroy(self):
        if self._h is not None:
            self._h.close()
        self._h = None
        self.setup_done = False

    def print_short(self):
        print(f"ILS solver : {self.name} -> it/maxit = {self.it:3d}/{self.maxit:3d} and "
              f"rerr/rcvg = {self.rerr:10.2e}/{self.rcvg:10.2e}")
