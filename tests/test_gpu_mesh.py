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


def _mesh_case():
    m = S.mesh_scene([(3, (1.0, 0.8, 0.6), (0.1, 0.2, 0.3), (0.0, 0.0, 0.0), 0.1),
                      (3, (0.7, 0.9, 0.5), (0.3, -0.2, 0.1), (2.6, 0.4, -0.2), 0.1)])
    Mo, rhs = O.mesh_operator(m["V"], m["F"], m["face_body"], m["body_pos"], m["S"])
    return m, Mo, rhs


def test_matrix_free_mesh_operator_products():
    """The matrix-free mesh operator (MBC_OP_MESH: solid angles evaluated in
    the matvec) against the oracle's dense FP64 matrix: K and K^T within 1e-12
    (FP64 solver) and 2e-5 (FP32 solver), norm-wise relative."""
    import fastmbcui_b200 as F

    m, Mo, _ = _mesh_case()
    d = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    plan = F.Plan(m["S"], 3.0, 1.5, 2048)
    rng = np.random.default_rng(0)
    V, W = rng.standard_normal((Mo.shape[1], 5)), rng.standard_normal((Mo.shape[0], 5))
    for prec, tol, dt in ((F.MBC_F64, 1e-12, torch.float64), (F.MBC_F32, 2e-5, torch.float32)):
        s = F.Solver(plan, mesh=(d(m["V"]), d(m["F"], torch.int32), d(m["S"])), precision=prec)
        got_k = s.apply_K(d(V, dt)).double().cpu().numpy()
        got_kt = s.apply_KT(d(W, dt)).double().cpu().numpy()
        assert np.linalg.norm(got_k - Mo @ V) / np.linalg.norm(Mo @ V) < tol
        assert np.linalg.norm(got_kt - Mo.T @ W) / np.linalg.norm(Mo.T @ W) < tol


def test_matrix_free_mesh_operator_solve_matches_oracle():
    """Factor and PCG with the matrix-free mesh operator against the oracle
    on the same FP64 dense matrix: the KL factor within 1e-7 per column
    (norm-wise), PCG iterations within max(3, 3 %) per column, and the FP64
    true residual (dense oracle matrix) <= tol."""
    import fastmbcui_b200 as F

    m, Mo, rhs = _mesh_case()
    d = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    plan = F.Plan(m["S"], 3.0, 1.5, 2048)
    pl = O.plan(m["S"], 3.0, 1.5, 2048)
    op = O.Op(Mo.shape[0], Mo.shape[1], M=Mo)
    _, lval_o, _ = O.factor(op, pl)
    s = F.Solver(plan, mesh=(d(m["V"]), d(m["F"], torch.int32), d(m["S"])), precision=F.MBC_F64).factor()
    lval, _ = s.get_factor()
    lp = pl["lptr"]
    for c in range(0, Mo.shape[1], max(1, Mo.shape[1] // 50)):
        a, b = lp[c], lp[c + 1]
        assert np.linalg.norm(lval[a:b] - lval_o[a:b]) <= 1e-7 * np.linalg.norm(lval_o[a:b])
    cols = [c for c in range(rhs.shape[1]) if np.linalg.norm(rhs[:, c]) > 0]
    X, st, its = s.solve(d(rhs[:, cols], torch.float64), tol=1e-8, max_iters=4000, iters=True)
    X = X.cpu().numpy()
    for k, c in enumerate(cols):
        xo, it, _ = O.pcg(op, pl, lval_o, f=rhs[:, c], maxits=4000, tol=1e-8)
        assert abs(int(its[k]) - it) <= max(3, 0.03 * it), (c, int(its[k]), it)
        b = Mo.T @ rhs[:, c]
        r = Mo.T @ (rhs[:, c] - Mo @ X[:, k])
        assert np.linalg.norm(r) <= 1.05e-8 * np.linalg.norm(b)
