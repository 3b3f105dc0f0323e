"""Flexible conjugate gradients in FP64 around an FP32 inner PCG.

On the ill-conditioned normal equations of MFS, an FP32 operator cannot
drive the FP64 residual to 1e-8: residual replacement stalls and the
restarted FP64 polish throws the Krylov space away.  Here the FP32 PCG
(tensor-core matvec, FP32 KL preconditioner, a fixed number of iterations)
is the *preconditioner* of an FP64 flexible CG (Notay's FCG): each outer step
applies the FP64 operator once, orthogonalises the inner solution against the
last ``keep`` search directions in the FP64 operator's inner product, and
updates x and r in FP64.  The outer recursion keeps what the inner solves
learn, so the FP64 matvec count drops by an order of magnitude.

``flexible_cg`` is written on array operations only (torch tensors, any
device), with the operator and the inner solve passed in; ``solve_flexible``
binds them to two solvers of libmbc (FP64 and FP32) on the same plan.
"""
from __future__ import annotations


def _colsum(a):
    return a.sum(dim=0)


def flexible_cg(apply64, inner, b, tol=1e-8, keep=20, max_outer=300, check_true=True, x0=None):
    """Solve A X = B column by column (batched), A symmetric positive definite.

    apply64(V) -> A V (FP64, n x R); inner(R) -> an approximation of A^-1 R for
    columns scaled to unit norm.  x0: a starting point (costs one more FP64
    application).  Stops a column when |r| <= tol |b|; with check_true the
    recursive residual is confirmed by b - A x before stopping (and replaces r
    if it had drifted).  Returns (X, info)."""
    import torch

    n_apply, n_outer, n_replace = 0, 0, 0
    if x0 is None:
        x = torch.zeros_like(b)
        r = b.clone()
    else:
        x = x0.to(b.dtype).clone()
        r = b - apply64(x)
        n_apply += 1
    bn = torch.linalg.norm(b, dim=0)
    P, Q, PQ = [], [], []
    for k in range(max_outer):
        rn = torch.linalg.norm(r, dim=0)
        done = rn <= tol * bn
        if bool(done.all()) and check_true:
            rt = b - apply64(x)
            n_apply += 1
            rtn = torch.linalg.norm(rt, dim=0)
            if bool((rtn <= tol * bn).all()):
                r = rt
                break
            # the recursion drifted: restart the residual from the true one
            r = rt
            n_replace += 1
            P, Q, PQ = [], [], []
            continue
        if bool(done.all()):
            break
        scale = torch.where(done, torch.zeros_like(rn), 1.0 / torch.where(rn > 0, rn, torch.ones_like(rn)))
        z = inner(r * scale)
        # finished columns take no step, whatever the inner solve returned for
        # their zero right-hand side
        z = torch.where(done, torch.zeros_like(z), z * rn)
        for p, q, pq in zip(P, Q, PQ):
            z = z - p * (_colsum(z * q) / pq)
        q = apply64(z)
        n_apply += 1
        zq = _colsum(z * q)
        ok = (~done) & (zq > 0)
        alpha = torch.where(ok, _colsum(z * r) / torch.where(ok, zq, torch.ones_like(zq)), torch.zeros_like(zq))
        x = x + alpha * z
        r = r - alpha * q
        P.append(z)
        Q.append(q)
        PQ.append(torch.where(ok, zq, torch.ones_like(zq)))
        if len(P) > keep:
            P.pop(0)
            Q.pop(0)
            PQ.pop(0)
        n_outer += 1
    rel = torch.linalg.norm(r, dim=0) / torch.where(bn > 0, bn, torch.ones_like(bn))
    return x, {"outer": n_outer, "fp64_applies": n_apply, "replacements": n_replace,
               "relres_max": float(rel.max()), "converged": int((rel <= tol).sum())}


def solve_flexible(s64, s32, F, tol=1e-8, inner_iters=40, keep=20, max_outer=300, adjoint=False, X0=None,
                   profile=False):
    """Forward solve (K^T K) X = K^T F (or, with adjoint, (K^T K) X = F) with
    FP64 flexible CG around the FP32 solver's plain PCG.

    s64, s32: solvers of the same plan and operator, precision FP64 and FP32;
    s32 factored (its KL factor preconditions the inner PCG), s64 used only
    for operator applications.  X0: optional n x R start (original order).
    Returns (X float64, n x R, original order; info).  info adds the FP32
    inner iterations and library kernel launches and, with profile, the
    CUDA-event time of the FP64 applications and of the inner matvecs."""
    import torch

    from . import MBC_FP64_MATVEC_INT8

    F = F if F.dim() == 2 else F[:, None]
    F64 = F.double().contiguous()
    b = F64 if adjoint else s64.apply_KT(F64)
    # kernels per FP64 direction: one CUDA-core kernel, or pack + MMA on the INT8 path
    per_dir = 2 if getattr(s64, "fp64_matvec", 0) == MBC_FP64_MATVEC_INT8 else 1
    acc = {"inner": 0, "launches": (per_dir + 1) if not adjoint else 0, "t64": 0.0, "n64": 0, "t32": 0.0,
           "n32": 0}

    def apply64(v):
        if profile:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        out = s64.apply_KT(s64.apply_K(v.contiguous()))
        if profile:
            e1.record()
            e1.synchronize()
            acc["t64"] += e0.elapsed_time(e1)
        acc["n64"] += 2
        acc["launches"] += 2 + 2 * per_dir  # permute, K, K^T, permute
        return out

    def inner(rs):
        z, st = s32.solve_adjoint(rs.float().contiguous(), out_dtype=torch.float32, tol=0.0,
                                  max_iters=inner_iters, max_refine=0, profile=1 if profile else 0)
        acc["inner"] += int(st["iters_max"])
        acc["launches"] += int(st["kernel_launches"])
        acc["t32"] += float(st["t_matvec_ms"])
        acc["n32"] += int(st["n_matvec"])
        return z.double()

    X, info = flexible_cg(apply64, inner, b, tol=tol, keep=keep, max_outer=max_outer,
                          x0=None if X0 is None else X0.double())
    info.update({"fp32_inner_iterations": acc["inner"], "kernel_launches": acc["launches"],
                 "t_matvec64_ms": acc["t64"], "n_matvec64": acc["n64"], "t_matvec32_ms": acc["t32"],
                 "n_matvec32": acc["n32"]})
    return X, info


__all__ = ["flexible_cg", "solve_flexible"]
