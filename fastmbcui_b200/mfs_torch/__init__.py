"""Drop-in for the reference's ``mfs_torch`` operator package.

The reference loads ``./build/mfs_torch/csrc/libmfs_torch.so`` and exposes
``mfs.ops.MinvF_float_fastGrad`` (core/mfs_torch_py/__init__.py:7-10).
Importing this package registers the same two operators,

    mfs_torch::MinvF_float_fastGrad(Tensor M, Tensor F, Tensor Vs_s, float rho,
        int pcg_max_iter, float tol_r, bool timing_verbose=False,
        bool solve_verbose=False) -> Tensor
    mfs_torch::VpL_fast_float(Tensor M, Tensor pL, Tensor Vs_s, float rho,
        int pcg_max_iter, float tol_r, bool timing_verbose=False,
        bool solve_verbose=False) -> Tensor

(mfs_torch/csrc/mfs_torch_ops.cpp:8-9), backed by libmbc.so, so a caller
switches with ``import fastmbcui_b200.mfs_torch as mfs``.
"""
from . import ops  # noqa: F401  (registers the operators)

__all__ = ["ops"]
