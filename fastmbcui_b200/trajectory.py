"""Solving a moving scene step after step.

A rigid-body simulation calls the MFS solve once per time step
(core/KTAB_Mfs_spclf1d.py:117, one MinvF_float_fastGrad call per
compute_kirchhoff_tensor) on bodies that moved a little since the last step.
``TrajectorySolver`` is that call for point-kernel scenes: every step builds a
new supernodal factor on the current geometry, solves all rigid-mode columns
in one batched PCG to the FP64 tolerance, and starts from the strengths of the
previous steps instead of x0 = 0 (the reference always starts from zero,
src/kl_chol.cu:930-940).

Precision modes (``mode``):
  "mixed"  the factor and its application in FP32 (supernodes whose FP32
           Cholesky cancels are refactored in FP64); the PCG recursion,
           dot products and scalars in FP64; the matvecs FP64-accurate
           (``fp64_matvec="int8"``: exact digit slices on the INT8 tensor
           cores, or "simt": FP64 CUDA cores).
  "fp64"   the plain method: FP64 factor and FP64 PCG.
  "fp32-replace"  FP32 recursion (tensor-core 3xTF32 matvec) with FP64
           residual replacement and an FP64 polish of stagnating columns.

Schedules (``schedule``): "block" (block PCG: the columns share one Krylov
space, so slowly converging columns borrow the directions the others found;
"mixed" and "fp64" modes) or "batched" (independent per-column recurrences
advanced together).

Factor tile shapes (``factor_tiles``): a dict for mbc_solver_set_factor_tiles,
None for the library's defaults, or "tuned" (the default): the table the
autotuner (fastmbcui_b200.tune_factor) picked on the 32-ellipsoid trajectory
scene, data/factor_tiles_b200.json, when present.

Ordering reuse (``plan_every``): the host plan (maximin ordering, pattern,
supernodes) of a step is rebuilt every ``plan_every`` steps (1, the default,
is the plain method: a new plan per call, as mfs_torch_ops.cu:51-55 and
:114-116 build one); with K > 1 the plan of a step is reused for the next
K - 1 steps of slowly moving bodies while the factor is always rebuilt on the
current geometry.  That changes the preconditioner, not the solution, which
every column's own FP64 residual still decides.

Warm starts (``warm``): "extrapolate" (quadratic extrapolation of the last
three steps' strengths, linear with two, the previous with one), "previous",
"cold" (x0 = 0), or a callable ``warm(history) -> X0 or None``.
Every column is still decided on its own FP64 residual, whatever the start.
"""
from __future__ import annotations

import json
import os

from . import MBC_F32, MBC_F64, MBC_SCHED_BATCHED, MBC_SCHED_BLOCK, Solver

MODES = ("mixed", "fp64", "fp32-replace")
TUNED_TILES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "factor_tiles_b200.json")


def tuned_tiles():
    """The committed autotuner table, or None."""
    try:
        with open(TUNED_TILES) as f:
            return json.load(f)["tiles"]
    except (OSError, KeyError, ValueError):
        return None


def extrapolate(hist):
    """x0 from the strengths of the previous steps (newest last)."""
    if not hist:
        return None
    if len(hist) >= 3:
        return 3.0 * hist[-1] - 3.0 * hist[-2] + hist[-3]
    if len(hist) == 2:
        return 2.0 * hist[-1] - hist[-2]
    return hist[-1]


class TrajectorySolver:
    def __init__(self, coef: float, *, mode: str = "mixed", fp64_matvec: str = "int8",
                 warm="extrapolate", tol: float = 1e-8, max_iters: int = 3000, check_every: int = 8,
                 compact: bool = False, matvec: int = 0, schedule: str = "block", factor_tiles="tuned",
                 plan_every: int = 1):
        if mode not in MODES:
            raise ValueError(f"mode must be one of {MODES}")
        self.coef, self.mode, self.fp64_matvec = float(coef), mode, fp64_matvec
        self.warm, self.tol, self.max_iters = warm, float(tol), int(max_iters)
        self.check_every, self.compact, self.matvec = int(check_every), bool(compact), int(matvec)
        self.schedule = {"block": MBC_SCHED_BLOCK, "batched": MBC_SCHED_BATCHED}[schedule]
        self.factor_tiles = tuned_tiles() if factor_tiles == "tuned" else factor_tiles
        if int(plan_every) < 1:
            raise ValueError("plan_every must be >= 1")
        self.plan_every = int(plan_every)
        self._plan, self._plan_age = None, 0
        self.history = []

    def plan_for(self, pts, rho: float, lam: float, max_super: int):
        """The host plan for this step's source points (n x 3): a new one
        every plan_every steps, else the last one."""
        from . import Plan

        if self._plan is None or self._plan_age >= self.plan_every:
            self._plan, self._plan_age = Plan(pts, rho, lam, max_super), 0
        self._plan_age += 1
        return self._plan

    def start(self):
        """The warm start of the next step (None: x0 = 0)."""
        if callable(self.warm):
            return self.warm(self.history)
        if self.warm == "cold" or not self.history:
            return None
        if self.warm == "previous":
            return self.history[-1]
        if self.warm == "extrapolate":
            return extrapolate(self.history)
        raise ValueError(f"unknown warm start {self.warm!r}")

    def solver(self, plan, x, nx, y):
        """A factored solver of this mode for one step's geometry."""
        if self.mode == "fp64":
            s = Solver(plan, x=x, nx=nx, y=y, coef=self.coef, precision=MBC_F64)
        else:
            s = Solver(plan, x=x, nx=nx, y=y, coef=self.coef, precision=MBC_F32)
            s.set_matvec(self.matvec)
        if self.factor_tiles:
            s.set_factor_tiles(self.factor_tiles)
        return s.set_fp64_matvec(self.fp64_matvec).factor()

    def step(self, plan, x, nx, y, F, *, X0=None, profile: int = 0, keep: bool = True):
        """Factor on this step's geometry and solve F (nf x R); returns
        (X (n x R, FP64 except in "fp32-replace" mode), stats).  The
        result joins the history the next warm start is formed from unless
        keep=False; X0 overrides the warm start."""
        import torch

        if X0 is None:
            X0 = self.start()
        s = self.solver(plan, x, nx, y)
        opts = dict(X0=X0, profile=profile, tol=self.tol, max_iters=self.max_iters,
                    check_every=self.check_every)
        if self.mode == "fp32-replace":
            X, st = s.solve(F, out_dtype=torch.float32, max_refine=64, inner_tol=1e-2,
                            compact=int(self.compact), **opts)
        else:
            X, st = s.solve(F, out_dtype=torch.float64, compact=int(self.compact), schedule=self.schedule,
                            fp64_recursion=1 if self.mode == "mixed" else 0, **opts)
        if keep:
            self.history = (self.history + [X])[-3:]
        return X, st
