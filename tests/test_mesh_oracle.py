"""The mesh collocation operator's CPU oracle.

* Against the golden fixture made by the reference's own torch functions
  (tests/golden/make_mesh_golden.py): 1e-13 relative.
* Gauss: the faces of a closed, outward-oriented surface subtend 4 pi at a
  point inside and 0 at a point outside; the area-weighted normals and their
  moments sum to zero over a closed surface.
"""
import os

import numpy as np

import oracle as O
from fastmbcui_b200 import scenes as S

GOLD = os.path.join(os.path.dirname(__file__), "golden", "mesh_two_bodies.npz")


def test_oracle_matches_reference_functions():
    z = np.load(GOLD)
    M, rhs = O.mesh_operator(z["V"], z["F"], z["face_body"], z["body_pos"], z["S"])
    assert np.abs(M - z["M"]).max() <= 1e-13 * np.abs(z["M"]).max()
    assert np.abs(rhs - z["FLIQ"]).max() <= 1e-13 * np.abs(z["FLIQ"]).max()


def test_solid_angles_close_to_4pi_inside_and_0_outside():
    V, F = S.icosphere_mesh(3)
    V = V * np.array([1.3, 0.9, 0.6])
    rng = np.random.default_rng(0)
    inside = rng.uniform(-0.3, 0.3, size=(20, 3))
    outside = np.array([[3.0, 0.0, 0.0], [0.0, -2.0, 1.0], [1.4, 0.0, 0.0]])
    M, rhs = O.mesh_operator(V, F, np.zeros(F.shape[0], np.int32), np.zeros((1, 3)),
                             np.concatenate([inside, outside]))
    tot = M.sum(axis=0)
    assert np.allclose(tot[:20], 4 * np.pi, rtol=0, atol=1e-11)
    assert np.abs(tot[20:]).max() < 1e-11
    # closed surface: sum of area-weighted normals and of their moments vanish
    area = np.linalg.norm(rhs[:, :3], axis=1).sum()
    assert np.abs(rhs.sum(axis=0)).max() < 1e-12 * area


def test_rhs_blocks_follow_the_bodies():
    z = np.load(GOLD)
    _, rhs = O.mesh_operator(z["V"], z["F"], z["face_body"], z["body_pos"], z["S"])
    for f in range(rhs.shape[0]):
        b = z["face_body"][f]
        other = np.delete(rhs[f].reshape(-1, 6), b, axis=0)
        assert np.all(other == 0.0)


FIXTURE_BODIES = [(1, (1.0, 0.7, 0.5), (0.3, -0.5, 0.2), (0.3, -0.2, 0.1), 0.1),
                  (1, (0.6, 0.6, 0.6), (-0.4, 0.1, 0.7), (2.6, 0.4, -0.3), 0.08)]


def test_mesh_scene_reproduces_fixture_inputs():
    # the package's own vertex normals place the sources exactly where the
    # reference's compute_normal_vertex put them for the fixture
    z = np.load(GOLD)
    m = S.mesh_scene(FIXTURE_BODIES)
    for k in ("V", "F", "face_body", "body_pos", "S"):
        assert np.array_equal(m[k], z[k]), k
