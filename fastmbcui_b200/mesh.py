"""The mesh collocation operator on the device (mbc_mesh_assemble).

The reference assembles, every step, the solid-angle collocation matrix of its
triangle meshes and the rigid-mode right-hand side in torch
(core/KTAB_Mfs_spclf1d.py:95-113); ``assemble`` builds both on the GPU, ready
for the ``mfs_torch`` operator (FP32) or for checks (FP64).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, load


def assemble(V, F, S, face_body=None, body_pos=None, dtype=None):
    """M (faces x sources): the solid angle of each face seen from each source;
    with face_body / body_pos also the right-hand side (faces x 6 bodies):
    per face (s, r x s), s its area-weighted normal, r its centre minus its
    body's position.  Inputs: array-likes (moved to the current CUDA device)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    dtype = dtype or torch.float32
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32) if isinstance(a, np.ndarray) else a,
                                    dtype=torch.float32, device=dev).contiguous()
    i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.int32) if isinstance(a, np.ndarray) else a,
                                    dtype=torch.int32, device=dev).contiguous()
    V, F, S = f32(V), i32(F), f32(S)
    nfc, ns = F.shape[0], S.shape[0]
    M = torch.empty((nfc, ns), dtype=dtype, device=dev)
    rhs = fb = bp = None
    nb = 0
    if face_body is not None:
        fb, bp = i32(face_body), f32(body_pos)
        nb = bp.shape[0]
        rhs = torch.empty((nfc, 6 * nb), dtype=dtype, device=dev)
    dt = _lib.MBC_F64 if dtype == torch.float64 else _lib.MBC_F32
    ptr = lambda t: None if t is None else t.data_ptr()
    check(load().mbc_mesh_assemble(V.shape[0], V.data_ptr(), nfc, F.data_ptr(), ptr(fb), nb, ptr(bp), ns,
                                   S.data_ptr(), dt, M.data_ptr(), ns, ptr(rhs),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)), "mbc_mesh_assemble")
    return (M, rhs) if rhs is not None else M
