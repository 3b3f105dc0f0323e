"""The ``mfs_torch`` operators on libmbc.so (schemas, checks, fakes, autograd).

Mirrors core/mfs_torch_py/ops.py:7-71 and the argument checks of
mfs_torch/csrc/mfs_torch_ops.cu:24-33 and :202-215.  The CUDA kernels are
libmbc's (mbc_minvf_float / mbc_vpl_fast_float); there is no CPU kernel, so a
CPU-tensor call fails in the dispatcher exactly as with the reference.
"""
from __future__ import annotations

import ctypes as C

import torch
from torch import Tensor

from .. import _lib

__all__ = ["MinvF_float_fastGrad", "VpL_fast_float"]

_SCHEMA_TAIL = ("Tensor Vs_s, float rho, int pcg_max_iter, float tol_r, "
                "bool timing_verbose=False, bool solve_verbose=False) -> Tensor")

_lib.load()  # fail loudly when libmbc.so is missing

_defined = False


def _define():
    global _defined
    if _defined:
        return
    torch.library.define("mfs_torch::VpL_fast_float", "(Tensor M, Tensor pL, " + _SCHEMA_TAIL)
    torch.library.define("mfs_torch::MinvF_float_fastGrad", "(Tensor M, Tensor F, " + _SCHEMA_TAIL)
    _defined = True


_define()

# One context per device: the explicit form of the reference's static factor
# cache (mfs_torch_ops.cu:17-19); VpL reuses the factor of the last forward.
_contexts: dict = {}


def _context(dev: torch.device):
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    h = _contexts.get(idx)
    if h is None:
        h = C.c_void_p()
        _lib.check(_lib.load().mbc_context_create(C.byref(h)), "mbc_context_create")
        _contexts[idx] = h
    return h


def _common_checks(M, R, Vs_s, rhs_name):
    torch._check(M.dtype == torch.float, lambda: "M must be float32")
    torch._check(R.dtype == torch.float, lambda: f"{rhs_name} must be float32")
    torch._check(Vs_s.dtype == torch.float, lambda: "Vs_s must be float32")
    torch._check(M.device.type == "cuda", lambda: "M must be a CUDA tensor")
    torch._check(R.device.type == "cuda", lambda: f"{rhs_name} must be a CUDA tensor")
    torch._check(Vs_s.device.type == "cpu", lambda: "Vs_s must be a CPU tensor")


def _run(fn, M, R, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose, solve_verbose):
    M = M.contiguous()
    R = R.contiguous()
    Vs = Vs_s.contiguous()
    n, k = M.shape[1], R.shape[1]
    out = torch.empty((n, k), dtype=torch.float, device=M.device)
    with torch.cuda.device(M.device):
        stream = torch.cuda.current_stream(M.device).cuda_stream
        s = getattr(_lib.load(), fn)(_context(M.device), M.data_ptr(), M.shape[0], n, R.data_ptr(), k,
                                     Vs.data_ptr(), float(rho), int(pcg_max_iter), float(tol_r),
                                     int(bool(timing_verbose)), int(bool(solve_verbose)),
                                     out.data_ptr(), C.c_void_p(stream))
    _lib.check(s, fn)
    return out


@torch.library.impl("mfs_torch::MinvF_float_fastGrad", "CUDA")
def _minvf_cuda(M, F, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose=False, solve_verbose=False):
    torch._check(F.dim() == 2, lambda: "F must be a 2D tensor")
    torch._check(M.size(0) == F.size(0), lambda: "M and F must have the same first dimension")
    torch._check(M.size(1) == Vs_s.size(0), lambda: "M and Vs_s must have compatible dimensions")
    torch._check(Vs_s.size(1) == 3, lambda: "Vs_s must be 3d points")
    _common_checks(M, F, Vs_s, "F")
    return _run("mbc_minvf_float", M, F, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose, solve_verbose)


@torch.library.impl("mfs_torch::VpL_fast_float", "CUDA")
def _vpl_cuda(M, pL, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose=False, solve_verbose=False):
    torch._check(pL.dim() == 2, lambda: "pL must be a 2D tensor")
    torch._check(M.size(1) == pL.size(0), lambda: "M and pL must have compatible dimensions")
    torch._check(M.size(1) == Vs_s.size(0), lambda: "M and Vs_s must have compatible dimensions")
    torch._check(Vs_s.size(1) == 3, lambda: "Vs_s must be 3d points")
    _common_checks(M, pL, Vs_s, "pL")
    return _run("mbc_vpl_fast_float", M, pL, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose,
                solve_verbose)


def MinvF_float_fastGrad(M: Tensor, F: Tensor, Vs_s: Tensor, rho: float, pcg_max_iter: int, tol_r: float,
                         timing_verbose: bool = False, solve_verbose: bool = False) -> Tensor:
    """Performs M.pinv @ F (least squares per column via PCG on the normal equations)."""
    return torch.ops.mfs_torch.MinvF_float_fastGrad.default(M, F, Vs_s, rho, pcg_max_iter, tol_r,
                                                          timing_verbose, solve_verbose)


def VpL_fast_float(M: Tensor, pL: Tensor, Vs_s: Tensor, rho: float, pcg_max_iter: int, tol_r: float,
                   timing_verbose: bool = False, solve_verbose: bool = False) -> Tensor:
    """Solves (M^T M) X = pL with the factor of the last forward on the same inputs."""
    return torch.ops.mfs_torch.VpL_fast_float.default(M, pL, Vs_s, rho, pcg_max_iter, tol_r,
                                                    timing_verbose, solve_verbose)


@torch.library.register_fake("mfs_torch::MinvF_float_fastGrad")
def _(M, F, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose=False, solve_verbose=False):
    torch._check(M.shape[0] == F.shape[0])
    torch._check(M.shape[1] == Vs_s.shape[0])
    torch._check(Vs_s.shape[1] == 3)
    torch._check(M.dtype == torch.float)
    torch._check(F.dtype == torch.float)
    torch._check(Vs_s.dtype == torch.float)
    torch._check(M.device == F.device)
    return torch.empty([Vs_s.shape[0], F.shape[1]], dtype=torch.float, device=M.device)


@torch.library.register_fake("mfs_torch::VpL_fast_float")
def _(M, pL, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose=False, solve_verbose=False):
    torch._check(M.shape[1] == pL.shape[0])
    torch._check(M.shape[1] == Vs_s.shape[0])
    torch._check(Vs_s.shape[1] == 3)
    torch._check(M.dtype == torch.float)
    torch._check(pL.dtype == torch.float)
    torch._check(Vs_s.dtype == torch.float)
    torch._check(M.device == pL.device)
    return torch.empty([Vs_s.shape[0], pL.shape[1]], dtype=torch.float, device=M.device)


def _setup_context(ctx, inputs, output):
    M, F, Vs_s, rho, pcg_max_iter, tol_r, timing_verbose, solve_verbose = inputs
    if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
        saved = (M, F, Vs_s, output)
        ctx.rho, ctx.pcg_max_iter, ctx.tol_r = rho, pcg_max_iter, tol_r
        ctx.timing_verbose, ctx.solve_verbose = timing_verbose, solve_verbose
    else:
        saved = (None, None, None, None)
    ctx.save_for_backward(*saved)


def _backward(ctx, grad):
    """grad_M = -M (W + W^T) + F LV, grad_F = M VpL (core/mfs_torch_py/ops.py:42-58),
    W = A LV, LV = VpL^T; computed in the equal low-rank form
    grad_M = (F - M A) VpL^T - (M VpL) A^T by the library's kernels
    (mbc_minvf_grad), without the N x N matrix W."""
    grad_M, grad_F = None, None
    if not (ctx.needs_input_grad[0] or ctx.needs_input_grad[1]):
        return grad_M, grad_F, None, None, None, None, None, None
    M, F, Vs_s, A = ctx.saved_tensors
    VpL = torch.ops.mfs_torch.VpL_fast_float.default(M, grad, Vs_s, ctx.rho, ctx.pcg_max_iter,
                                                     ctx.tol_r, ctx.timing_verbose,
                                                     ctx.solve_verbose)
    M, F, A, VpL = (t.contiguous() for t in (M, F, A, VpL))
    nf, n = M.shape
    R = A.shape[1]
    work = torch.empty((nf, 2 * R), dtype=torch.float32, device=M.device)
    if ctx.needs_input_grad[0]:
        grad_M = torch.empty_like(M)
    if ctx.needs_input_grad[1]:
        grad_F = torch.empty_like(F)
    st = C.c_void_p(torch.cuda.current_stream(M.device).cuda_stream)
    _lib.check(_lib.load().mbc_minvf_grad(nf, n, R, M.data_ptr(), M.stride(0), F.data_ptr(), A.data_ptr(),
                                          VpL.data_ptr(), work.data_ptr(),
                                          None if grad_M is None else grad_M.data_ptr(), n,
                                          None if grad_F is None else grad_F.data_ptr(), st),
               "mbc_minvf_grad")
    return grad_M, grad_F, None, None, None, None, None, None


torch.library.register_autograd("mfs_torch::MinvF_float_fastGrad", _backward,
                                setup_context=_setup_context)
