"""Autotune the factor kernels' tile shapes on the 32-ellipsoid trajectory
scene (32 ellipsoids x 2000 points, N = Nf = 64000, the trajectory's first
pose) with the library's own tuner (mbc_solver_tune_factor), for the FP32
factor the trajectory solver uses, and write the table
fastmbcui_b200/data/factor_tiles_b200.json:

    python -m fastmbcui_b200.tune_factor [reps]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    import torch

    import fastmbcui_b200 as F
    from fastmbcui_b200 import scenes as S

    reps = int(sys.argv[1]) if len(sys.argv) > 1 else 3
    base, q, _ = S.trajectory_scene(32, 2000, seed=4, steps=500)
    sc = S.moved(base, q[0])
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, x=t(sc.x), nx=t(sc.nx), y=t(sc.y), coef=sc.coef, precision=F.MBC_F32)
    default = s.factor_tiles()
    s.factor()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms_default = []
    for _ in range(reps):
        ev0.record()
        s.factor()
        ev1.record()
        torch.cuda.synchronize()
        ms_default.append(ev0.elapsed_time(ev1))
    tiles, ms = s.tune_factor(reps)
    rec = {"scene": "32 ellipsoids x 2000 points, trajectory seed 4, pose 0 (N = Nf = 64000)",
           "precision": "FP32 factor (FP64 retry of cancelling supernodes)", "device": torch.cuda.get_device_name(),
           "tiles": tiles, "factor_ms": round(ms, 2), "default_tiles": default,
           "default_factor_ms": round(float(np.median(ms_default)), 2), "reps": reps}
    with open(os.path.join(HERE, "data", "factor_tiles_b200.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
