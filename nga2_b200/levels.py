"""Per-level device times of the V-cycle (``python -m nga2_b200.levels``).

Sets up the solver on one of the package's synthetic problems and prints, as
one JSON line, the device milliseconds of ``cycle(n)`` for every level n (the
V-cycle from level n down, the fused coarse tail included) and of the single
passes (a Gauss-Seidel sweep, residual, restriction, prolongation) on the
finest levels, then one full solve.  ``cycle(n) - cycle(n+1)`` is the cost of
level n within a V-cycle.  With ``--cycle N`` only cycle(N) runs, ``--reps``
times, which is the small case to put under a profiler.  With ``--setup`` it
times the setup (the whole Galerkin hierarchy) from a device-resident
operator instead, the call the two-phase solvers make on every density change.
"""
from __future__ import annotations

import argparse
import json

from . import bbmg as B
from . import problems as P


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--problem", choices=("drops", "periodic"), default="drops")
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--cycle", type=int, default=0, help="run only cycle(N)")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--setup", action="store_true", help="time bbmg_setup from a device operator")
    a = ap.parse_args(argv)
    n = a.n
    if a.problem == "periodic":
        pb = P.periodic_poisson(n, seed=1)
    else:
        pb = P.drops_poisson(n, seed=2024, rmin=6.0 * n / 256, rmax=20.0 * n / 256)
    prec = B.MIXED if a.precision == "mixed" else B.FP64
    pf = 1 if prec == B.MIXED else 0
    g = B.BBMG(n, n, n, pb.xper, pb.yper, pb.zper, method=B.PCG_BBOX, precision=prec)
    g.setup(pb.stc, pb.opr)
    if a.setup:
        import torch
        dopr = torch.from_numpy(pb.opr).cuda()
        ms = []
        for _ in range(a.reps):
            g.setup(pb.stc, dopr)
            ms.append(g.info["setup_ms"])
        ms.sort()
        print(json.dumps({"n": n, "precision": a.precision, "setup_ms_median": ms[len(ms) // 2],
                          "setup_ms_min": ms[0]}))
        g.close()
        return
    if a.cycle:
        print(json.dumps({"n": n, "cycle": a.cycle, "ms": g.profile("cycle", a.cycle, 0, pf, a.reps)}))
        g.close()
        return
    inf = g.info
    r = {"n": n, "problem": a.problem, "precision": a.precision, "dims": inf["level_dims"]}
    for lv in range(1, inf["nlvl"] + 1):
        r[f"cycle{lv}"] = round(g.profile("cycle", lv, 0, pf, a.reps), 4)
    for lv in range(1, min(3, inf["nlvl"] - 1) + 1):
        for st in ("relax", "residual", "restrict", "prolong"):
            r[f"{st}{lv}"] = round(g.profile(st, lv, 1, pf, a.reps), 4)
    for _ in range(2):
        _, it, rerr, st = g.solve(pb.rhs)
    r["solve_ms"] = round(g.info["solve_ms"], 3)
    r["it"] = it
    print(json.dumps(r))
    g.close()


if __name__ == "__main__":
    main()
