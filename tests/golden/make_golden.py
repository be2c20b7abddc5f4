"""Generates the committed golden fixtures of the bbmg oracle.

    python -m tests.golden.make_golden

Each fixture holds a seeded problem's hash, the oracle's solution, iteration
count and residual ratio.  The problems come from nga2_b200/problems.py with
fixed seeds; the solution is the CPU oracle's (oracle/bbmg_oracle.c, parity
build).  The periodic fixture is also checked against the exact FFT solution
when it is made.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from nga2_b200 import problems as P  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
BBOX, PCG_BBOX = 1, 2


def make_case(name):
    if name == "periodic16":
        return P.periodic_poisson(16, seed=4), BBOX
    if name == "walls16":
        stc, opr = P.random_operator(16, 12, 10, (True, False, True), seed=6)
        rng = np.random.default_rng(6)
        rhs = rng.standard_normal((10, 12, 16))
        rhs -= rhs.mean()
        vol = np.ones_like(rhs)
        return P.Problem("walls16", 16, 12, 10, True, False, True, stc, opr, rhs, vol, 6), PCG_BBOX
    if name == "drops24":
        return P.drops_poisson(24, seed=8, ndrops=4, rmin=2.0, rmax=4.0), PCG_BBOX
    raise KeyError(name)


def problem_sha(pb):
    h = hashlib.sha256()
    for a in (pb.stc, pb.opr, pb.rhs):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    from oracle.oracle import OracleBBMG, fft_solve_periodic
    for name in ("periodic16", "walls16", "drops24"):
        pb, method = make_case(name)
        o = OracleBBMG(pb.nx, pb.ny, pb.nz, pb.xper, pb.yper, pb.zper, method=method, rcvg=1e-10)
        o.setup(pb.stc, pb.opr)
        x, it, rerr = o.solve(pb.rhs)
        if name == "periodic16":
            ex = fft_solve_periodic(pb.opr, pb.rhs)
            err = np.abs(P.remove_mean(x) - ex).max() / np.abs(ex).max()
            assert err < 1e-8, err
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), sol=x, it=it, rerr=rerr,
                            problem_sha=problem_sha(pb), method=method)
        print(name, it, rerr)


if __name__ == "__main__":
    main()
