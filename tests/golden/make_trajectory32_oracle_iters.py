"""Measure, with the CPU oracle, the plain method's PCG iterations on the
32-ellipsoid trajectory scene (first pose, trajectory seed 4: 32 ellipsoids x
2000 points, N = Nf = 64000, R = 192, rho 3, lambda 1.5, tol 1e-8, x0 = 0),
and store them as a fixture:

    python tests/golden/make_trajectory32_oracle_iters.py [columns...]

The oracle's own FP64 plan, KL factor and PCG (orc_pcg_many: orc_pcg's
per-column recurrence, kl_chol.cu:891-1088, with the K / K^T passes shared
by the columns) run on a sample of the 192 rigid-mode columns, one per mode
type by default.  A full pass of K and K^T at this size takes seconds on a
few host cores, so the whole run takes hours; the result is committed so the
reference arm of the benchmark can use measured iteration counts, and the GPU
tests compare the library's plain FP64 path against them.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from fastmbcui_b200 import scenes as S  # noqa: E402

OUT = os.path.join(HERE, "trajectory32_oracle_iters.json")
# one column of each rigid mode (tx, ty, tz, rx, ry, rz), bodies spread over the scene
DEFAULT_COLS = [0, 43, 80, 117, 154, 191]


def main():
    cols = [int(c) for c in sys.argv[1:]] or DEFAULT_COLS
    O.build()
    base, q, _ = S.trajectory_scene(32, 2000, seed=4, steps=500)
    sc = S.moved(base, q[0])
    t0 = time.perf_counter()
    pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
    t_plan = time.perf_counter() - t0
    op = O.Op.from_scene(sc)
    t0 = time.perf_counter()
    _, lval, bad = O.factor(op, pl)
    t_fac = time.perf_counter() - t0
    print(f"plan {t_plan:.1f}s, factor {t_fac:.1f}s (bad pivots {bad})", flush=True)
    F = sc.rhs()[:, cols]
    t0 = time.perf_counter()
    _, its, rel = O.pcg_many(op, pl, lval, F, maxits=5000, tol=1e-8)
    t_pcg = time.perf_counter() - t0
    rec = {"scene": "trajectory seed 4, pose 0: 32 ellipsoids x 2000 points, N = Nf = 64000, R = 192",
           "rho": sc.rho, "lambda": sc.lam, "tol": 1e-8, "columns": cols,
           "iters": [int(v) for v in its], "relres": [float(v) for v in rel],
           "host_threads": O.num_threads(),
           "seconds": {"plan": round(t_plan, 1), "factor": round(t_fac, 1), "pcg": round(t_pcg, 1)},
           "pcg_seconds_per_iteration": round(t_pcg / max(1, int(its.max())), 3)}
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
