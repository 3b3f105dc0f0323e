"""Regenerate the mesh-operator golden fixture (run in a container with the reference).

Runs the REFERENCE's own torch functions from utils/torch_utils.py --
compute_normal_vertex (:4-47), compute_face_centers (:49-60),
compute_FL_matrix (:62-75) and compute_solid_angle (:306-334) -- in FP64 on
a two-body triangle-mesh scene whose coordinates are float32-exact, and
stores inputs and outputs, assembled as core/KTAB_Mfs_spclf1d.py:95-113
does (sources = vertices moved inward along the vertex normals; the
right-hand side FL @ IQ, block-diagonal over the bodies):

    python tests/golden/make_mesh_golden.py
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT]

from fastmbcui_b200 import scenes as S  # noqa: E402

# the reference tree (the directory holding utils/torch_utils.py): required,
# from the environment, with no default location
REF = os.environ.get("MBC_REFERENCE", "")


def _reference_utils():
    if not REF or not os.path.isfile(os.path.join(REF, "utils", "torch_utils.py")):
        raise SystemExit("set MBC_REFERENCE to the reference tree (the directory with utils/torch_utils.py)")
    spec = importlib.util.spec_from_file_location("ref_torch_utils", os.path.join(REF, "utils", "torch_utils.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def main():
    import torch

    U = _reference_utils()
    bodies = []
    # (subdivision, semi-axes, rotation vector, position, source offset)
    for subdiv, axes, rv, pos, off in ((1, (1.0, 0.7, 0.5), (0.3, -0.5, 0.2), (0.3, -0.2, 0.1), 0.1),
                                       (1, (0.6, 0.6, 0.6), (-0.4, 0.1, 0.7), (2.6, 0.4, -0.3), 0.08)):
        V, F = S.icosphere_mesh(subdiv)
        R = S.rotvec_matrix(rv)
        V = _f32((V * np.asarray(axes)) @ R.T + np.asarray(pos))
        N = U.compute_normal_vertex(V.copy(), F.astype(np.int64))
        Sb = _f32(V - off * N)
        bodies.append((V, F, _f32(pos), Sb))
    S_all = np.concatenate([b[3] for b in bodies])
    t = lambda a: torch.as_tensor(a, dtype=torch.float64)
    M = torch.cat([U.compute_solid_angle(t(V), torch.as_tensor(F, dtype=torch.int64), t(S_all))
                   for V, F, _, _ in bodies], dim=0).numpy()
    nb = len(bodies)
    n_faces = sum(b[1].shape[0] for b in bodies)
    FL = np.zeros((n_faces, 6 * nb))
    r0 = 0
    for b, (V, F, pos, _) in enumerate(bodies):
        Ft = torch.as_tensor(F, dtype=torch.int64)
        C = U.compute_face_centers(t(V), Ft)
        FLb = U.compute_FL_matrix(t(V), Ft, C - t(pos)).numpy()
        FL[r0:r0 + F.shape[0], 6 * b:6 * b + 6] = FLb
        r0 += F.shape[0]
    IQ6 = np.block([[np.zeros((3, 3)), np.eye(3)], [np.eye(3), np.zeros((3, 3))]])
    IQ = np.kron(np.eye(nb), IQ6)
    FLIQ = FL @ IQ
    voff = np.cumsum([0] + [b[0].shape[0] for b in bodies])
    Fg = np.concatenate([b[1] + voff[k] for k, b in enumerate(bodies)]).astype(np.int32)
    face_body = np.concatenate([np.full(b[1].shape[0], k, np.int32) for k, b in enumerate(bodies)])
    np.savez_compressed(os.path.join(HERE, "mesh_two_bodies.npz"),
                        V=np.concatenate([b[0] for b in bodies]).astype(np.float32), F=Fg, face_body=face_body,
                        body_pos=np.array([b[2] for b in bodies], np.float32), S=S_all.astype(np.float32),
                        M=M, FLIQ=FLIQ)
    print("wrote", M.shape, FLIQ.shape)


if __name__ == "__main__":
    main()
