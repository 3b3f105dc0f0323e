"""mbc_mesh_assemble (the mesh collocation operator on the GPU) against the
reference's own functions (golden fixture) and the CPU oracle.

Tolerances: FP64 output 1e-13 and FP32 output 1e-6 of the largest entry
(the kernel computes in FP64 from float32 coordinates); Gauss closure 1e-10.
"""
import os

import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLD = os.path.join(os.path.dirname(__file__), "golden", "mesh_two_bodies.npz")


def _rel_max(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-6)])
def test_matches_reference_functions(dtype, tol):
    from fastmbcui_b200 import mesh

    z = np.load(GOLD)
    M, rhs = mesh.assemble(z["V"], z["F"], z["S"], z["face_body"], z["body_pos"], dtype=dtype)
    assert M.dtype == dtype and M.shape == z["M"].shape and rhs.shape == z["FLIQ"].shape
    assert _rel_max(M.cpu().numpy(), z["M"]) < tol
    assert _rel_max(rhs.cpu().numpy(), z["FLIQ"]) < tol


def test_gauss_closure_on_finer_meshes():
    from fastmbcui_b200 import mesh

    m = S.mesh_scene([(4, (1.2, 0.8, 0.6), (0.2, 0.1, -0.3), (0.0, 0.0, 0.0), 0.05),
                      (3, (0.5, 0.5, 0.7), (0.0, 0.6, 0.1), (2.5, 0.3, 0.2), 0.05)])
    M = mesh.assemble(m["V"], m["F"], m["S"], dtype=torch.float64).cpu().numpy()
    for b in range(2):
        tot = M[m["face_body"] == b].sum(axis=0)
        assert np.abs(tot[m["src_body"] == b] - 4 * np.pi).max() < 1e-10
        assert np.abs(tot[m["src_body"] != b]).max() < 1e-10
    Mo, _ = O.mesh_operator(m["V"], m["F"], m["face_body"], m["body_pos"], m["S"])
    assert _rel_max(M, Mo) < 1e-13


def test_out_of_range_indices_give_nan_rows():
    from fastmbcui_b200 import mesh

    z = np.load(GOLD)
    F = z["F"].copy()
    F[7, 1] = z["V"].shape[0]  # a vertex that does not exist
    fb = z["face_body"].copy()
    fb[9] = 5  # a body that does not exist
    M, rhs = mesh.assemble(z["V"], F, z["S"], fb, z["body_pos"], dtype=torch.float64)
    M, rhs = M.cpu().numpy(), rhs.cpu().numpy()
    assert np.isnan(M[7]).all() and np.isfinite(np.delete(M, 7, axis=0)).all()
    assert np.isnan(rhs[7]).all() and np.isnan(rhs[9]).all()
    good = np.setdiff1d(np.arange(F.shape[0]), [7, 9])
    assert _rel_max(rhs[good], z["FLIQ"][good]) < 1e-13


def test_mesh_operator_feeds_the_drop_in_op():
    # M and the right-hand side from the GPU, solved by the mfs_torch operator;
    # the fitted flux agrees with the FP64 oracle's dense PCG (as in the
    # operator tests)
    import fastmbcui_b200.mfs_torch as mfs
    from fastmbcui_b200 import mesh

    z = np.load(GOLD)
    M, rhs = mesh.assemble(z["V"], z["F"], z["S"], z["face_body"], z["body_pos"], dtype=torch.float32)
    X = mfs.ops.MinvF_float_fastGrad(M, rhs, torch.as_tensor(z["S"]), 3.0, 2000, 1e-6).double().cpu().numpy()
    K = M.double().cpu().numpy()
    op = O.Op(K.shape[0], K.shape[1], M=K)
    pl = O.plan(z["S"].astype(np.float64), 3.0)
    _, lval, _ = O.factor(op, pl)
    R = rhs.double().cpu().numpy()
    for c in range(R.shape[1]):
        xo, _, _ = O.pcg(op, pl, lval, f=R[:, c], maxits=4000, tol=1e-6)
        d = np.linalg.norm(K @ X[:, c] - K @ xo[pl["P"]]) / np.linalg.norm(R[:, c])
        assert d < 1e-3, (c, d)
