"""Seeded synthetic MFS scenes.

A scene is what the MFS solve path of fastMBCUI consumes each time step
(core/KTAB_Mfs_spclf1d.py:97-117): boundary collocation points with outward
normals, point sources slightly inside each body, and one right-hand side per
rigid mode per body (normal velocity n.e_i and n.(e_i x (x - c))).  The
operator is the normal derivative of a Laplace point source,

    K(i, j) = coef * ((x_i - y_j) . n_i) / |x_i - y_j|^3,

which is src/kernels.h:24-40 (laplace_nm_3d_sl) scaled by ``coef``;
coef = -1/(4 pi) makes it the normal derivative of G = 1/(4 pi |x - y|).

Every coordinate is rounded to float32 (and held in float64 arrays), because
the reference's operator takes float32 source points and widens them to double
before ordering (mfs_torch/csrc/mfs_torch_ops.cu:44-46); keeping the inputs
float32-exact lets the FP64 and FP32 paths see the same geometry.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

COEF_LAPLACE_DN = -1.0 / (4.0 * np.pi)


def _f32(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).astype(np.float64))


@dataclass
class Scene:
    """Collocation rows ``x, nx`` (nf x 3), sources ``y`` (n x 3) and bodies."""

    name: str
    x: np.ndarray
    nx: np.ndarray
    y: np.ndarray
    row_body: np.ndarray
    src_body: np.ndarray
    centers: np.ndarray
    coef: float = COEF_LAPLACE_DN
    rho: float = 3.0
    lam: float = 1.5
    max_super: int = 2048
    tol: float = 1e-8
    meta: dict = field(default_factory=dict)

    @property
    def nf(self) -> int:
        return int(self.x.shape[0])

    @property
    def n(self) -> int:
        return int(self.y.shape[0])

    @property
    def n_bodies(self) -> int:
        return int(self.centers.shape[0])

    def moving_bodies(self) -> np.ndarray:
        """Bodies that get rigid-mode columns (all but meta["static"])."""
        static = set(int(b) for b in self.meta.get("static", ()))
        return np.array([b for b in range(self.n_bodies) if b not in static], dtype=np.int64)

    def rhs(self) -> np.ndarray:
        """Rigid-mode normal velocities, nf x 6*(moving bodies), float32-exact;
        the rows of static bodies (a fixed floor) are zero in every column."""
        mv = self.moving_bodies()
        f = np.zeros((self.nf, 6 * len(mv)), dtype=np.float64)
        for k, b in enumerate(mv):
            rows = np.nonzero(self.row_body == b)[0]
            n = self.nx[rows]
            r = self.x[rows] - self.centers[b]
            f[rows, 6 * k:6 * k + 3] = n
            f[rows, 6 * k + 3:6 * k + 6] = np.cross(r, n)
        return _f32(f)

    def body_ptr(self) -> np.ndarray:
        """Row offsets of the bodies (rows of body b are [ptr[b], ptr[b+1]))."""
        ptr = np.searchsorted(self.row_body, np.arange(self.n_bodies + 1)).astype(np.int32)
        if not np.array_equal(np.repeat(np.arange(self.n_bodies), np.diff(ptr)), self.row_body):
            raise ValueError("rows are not grouped by body")
        return ptr

    def weights(self) -> np.ndarray:
        """Quadrature weight of each collocation point: its body's area over
        its point count (the points are area-uniform samples)."""
        if "weights" in self.meta:
            return _f32(np.asarray(self.meta["weights"], dtype=np.float64))
        ptr = self.body_ptr()
        areas = np.asarray(self.meta["areas"], dtype=np.float64)
        w = np.repeat(areas / np.diff(ptr), np.diff(ptr))
        return _f32(w)

    def dense_K(self) -> np.ndarray:
        """Dense FP64 operator (nf x n); only for small scenes."""
        r = self.x[:, None, :] - self.y[None, :, :]
        r2 = (r[..., 0] * r[..., 0] + r[..., 1] * r[..., 1]) + r[..., 2] * r[..., 2]
        rn = (r[..., 0] * self.nx[:, None, 0] + r[..., 1] * self.nx[:, None, 1]) + r[..., 2] * self.nx[:, None, 2]
        return self.coef * rn / (np.sqrt(r2) * r2)


# --------------------------------------------------------------------------
# primitive surfaces (unit pose)
# --------------------------------------------------------------------------

def icosphere(subdiv: int) -> np.ndarray:
    """Unit icosphere vertices (10*4^subdiv + 2), deterministic order."""
    return icosphere_mesh(subdiv)[0]


def icosphere_mesh(subdiv: int):
    """Unit icosphere: vertices (10*4^subdiv + 2, deterministic order) and
    triangles (20*4^subdiv x 3, int32) ordered counter-clockwise seen from
    outside, so that (v1 - v0) x (v2 - v0) points outward."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache: dict = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int32)


def sample_cylinder(rng: np.random.Generator, npts: int, r: float, h: float):
    """Area-uniform points on a closed cylinder (axis z, centred); (p, n)."""
    a_side, a_cap = 2 * np.pi * r * h, np.pi * r * r
    probs = np.array([a_side, a_cap, a_cap]) / (a_side + 2 * a_cap)
    part = rng.choice(3, size=npts, p=probs)
    u, v = rng.random(npts), rng.random(npts)
    th = 2 * np.pi * u
    p = np.zeros((npts, 3))
    n = np.zeros((npts, 3))
    side = part == 0
    p[side] = np.stack([r * np.cos(th[side]), r * np.sin(th[side]), h * (v[side] - 0.5)], 1)
    n[side] = np.stack([np.cos(th[side]), np.sin(th[side]), np.zeros(side.sum())], 1)
    for k, zs in ((1, 0.5), (2, -0.5)):
        m = part == k
        rr = r * np.sqrt(v[m])
        p[m] = np.stack([rr * np.cos(th[m]), rr * np.sin(th[m]), np.full(m.sum(), zs * h)], 1)
        n[m] = np.array([0.0, 0.0, 1.0 if zs > 0 else -1.0])
    return p, n


def sample_ellipsoid(rng: np.random.Generator, npts: int, axes):
    """Area-uniform points on an ellipsoid by rejection from the sphere; (p, n)."""
    a, b, c = axes
    gmax = max(b * c, a * c, a * b)
    out = []
    need = npts
    while need > 0:
        u = rng.normal(size=(2 * need + 16, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        g = np.sqrt((b * c * u[:, 0]) ** 2 + (a * c * u[:, 1]) ** 2 + (a * b * u[:, 2]) ** 2)
        keep = u[rng.random(u.shape[0]) * gmax < g]
        out.append(keep[:need])
        need -= out[-1].shape[0]
    u = np.concatenate(out)[:npts]
    p = u * np.array([a, b, c])
    n = p / np.array([a * a, b * b, c * c])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return p, n


def ellipsoid_area(axes, n_theta: int = 2000) -> float:
    """Surface area of an ellipsoid by the midpoint rule in (theta, phi)."""
    a, b, c = (float(v) for v in axes)
    th = (np.arange(n_theta) + 0.5) * np.pi / n_theta
    ph = (np.arange(2 * n_theta) + 0.5) * np.pi / n_theta
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    sp, cp = np.sin(ph)[None, :], np.cos(ph)[None, :]
    g = st * np.sqrt((b * c * st * cp) ** 2 + (a * c * st * sp) ** 2 + (a * b * ct) ** 2)
    return float(g.sum() * (np.pi / n_theta) ** 2)


def sample_box(rng: np.random.Generator, npts: int, side: float):
    """Area-uniform points on a cube of edge ``side``; (p, n)."""
    face = rng.integers(0, 6, npts)
    uv = (rng.random((npts, 2)) - 0.5) * side
    p = np.zeros((npts, 3))
    n = np.zeros((npts, 3))
    for f in range(6):
        m = face == f
        ax, sg = f // 2, (1.0 if f % 2 == 0 else -1.0)
        o = [k for k in range(3) if k != ax]
        p[m, ax] = sg * side / 2
        p[m, o[0]] = uv[m, 0]
        p[m, o[1]] = uv[m, 1]
        n[m, ax] = sg
    return p, n


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def random_centers(rng: np.random.Generator, radii, box: float, margin: float = 0.1):
    """Rejection-sampled centres in [0, box]^3 whose bounding spheres do not touch."""
    cs: list = []
    for r in radii:
        for _ in range(100000):
            c = rng.random(3) * (box - 2 * r) + r
            if all(np.linalg.norm(c - d) > r + s + margin for d, s in cs):
                cs.append((c, r))
                break
        else:
            raise RuntimeError("could not place a body without overlap")
    return np.array([c for c, _ in cs])


def _assemble(name, parts, **kw) -> Scene:
    xs, ns, ys, rb, sb, cs = [], [], [], [], [], []
    for b, (p, n, src, c) in enumerate(parts):
        xs.append(p); ns.append(n); ys.append(src); cs.append(c)
        rb.append(np.full(p.shape[0], b, dtype=np.int32))
        sb.append(np.full(src.shape[0], b, dtype=np.int32))
    x = _f32(np.concatenate(xs))
    nx = np.concatenate(ns)
    nx = _f32(nx / np.linalg.norm(nx, axis=1, keepdims=True))
    return Scene(name=name, x=x, nx=nx, y=_f32(np.concatenate(ys)),
                 row_body=np.concatenate(rb), src_body=np.concatenate(sb),
                 centers=_f32(np.array(cs)), **kw)


# --------------------------------------------------------------------------
# the benchmark configurations
# --------------------------------------------------------------------------

def sphere_scene(subdiv: int = 4, src_radius: float = 0.8) -> Scene:
    """Plain MFS, single unit sphere: icosphere collocation, sources at 0.8.

    Subdivision 4 gives 2562 collocation points and 2562 sources; rho=3,
    lambda=1.5, PCG tolerance 1e-10.
    """
    v = icosphere(subdiv)
    return _assemble(f"sphere_ico{subdiv}", [(v, v, src_radius * v, np.zeros(3))],
                     rho=3.0, lam=1.5, tol=1e-10, meta={"areas": [4 * np.pi]})


def coins_scene(n_coins: int = 16, pts: int = 4000, offset: float = 0.02,
                sample_seed: int = 1, pose_seed: int = 2, box: float = 10.0) -> Scene:
    """Coins: cylinders r=1, h=0.1, area-sampled, sources `offset` inside.

    The offset defaults to 0.02: an inward offset of h/2 = 0.05 or more puts the
    sources of both caps in the mid-plane, where they cannot represent an
    antisymmetric cap flux, and the least-squares system stalls (relative
    normal-equation residual ~7e-4 after 2000 FP64 PCG iterations, against ~200
    iterations to 1e-8 at 0.02).
    """
    rs = np.random.default_rng(sample_seed)
    rp = np.random.default_rng(pose_seed)
    rad = float(np.hypot(1.0, 0.05))
    centers = random_centers(rp, [rad] * n_coins, box)
    parts = []
    for b in range(n_coins):
        p, n = sample_cylinder(rs, pts, 1.0, 0.1)
        R = random_rotation(rp)
        p, n = p @ R.T + centers[b], n @ R.T
        parts.append((p, n, p - offset * n, centers[b]))
    return _assemble(f"coins{n_coins}x{pts}", parts, rho=3.0, lam=1.5, tol=1e-8,
                     meta={"areas": [2 * np.pi * 0.1 + 2 * np.pi] * n_coins})


def ellipsoids_scene(n_bodies: int, pts, seed: int, box: float = 10.0,
                     offset: float = 0.05, axes_range=(0.5, 1.5)) -> Scene:
    """Random ellipsoids (semi-axes U[0.5,1.5]); sources `offset` inside along the normal.

    At 2000 points per body the point spacing is ~0.08; an offset of 0.05 keeps
    the system well posed (~130-220 FP64 PCG iterations to 1e-8 at rho=3),
    whereas sources at 0.8 of the centre distance stall near 1e-6.
    """
    rng = np.random.default_rng(seed)
    axes = rng.uniform(axes_range[0], axes_range[1], size=(n_bodies, 3))
    counts = np.broadcast_to(np.asarray(pts), (n_bodies,)) if np.ndim(pts) == 0 else np.asarray(pts)
    centers = random_centers(rng, axes.max(axis=1), box)
    parts = []
    for b in range(n_bodies):
        p, n = sample_ellipsoid(rng, int(counts[b]), axes[b])
        R = random_rotation(rng)
        p, n = p @ R.T, n @ R.T
        parts.append((p + centers[b], n, p - offset * n + centers[b], centers[b]))
    return _assemble(f"ellipsoids{n_bodies}", parts, rho=3.0, lam=1.5, tol=1e-8,
                     meta={"axes": axes, "areas": [ellipsoid_area(ax) for ax in axes]})


def large_scene(seed: int = 5, n_boxes: int = 20, box_pts: int = 5000, floor=(400, 250),
                spacing: float = 0.05, side_range=(0.3, 1.0)) -> Scene:
    """The large configuration: ``n_boxes`` boxes (edge U[0.3, 1], ``box_pts``
    area-uniform points each, random orientation) above a flat floor patch of
    400 x 250 collocation points on a square grid of ``spacing`` (normal +z).
    N = Nf = 200000 at the defaults, rho = 4, supernodes up to 512 wide.

    Sources sit 0.6 point spacings inside each box along the face normal and
    0.6 spacings below the floor (the ratio of the ellipsoid scenes, 0.05 /
    0.08).  Boxes do not touch one another (bounding spheres 0.1 apart) and
    clear the floor by 0.1.  The floor is static: rhs() has rigid-mode
    columns for the boxes only (R = 120 at the defaults).  Body n_boxes is
    the floor; its "center" is the patch centre."""
    rng = np.random.default_rng(seed)
    nxg, nyg = floor
    Lx, Ly = (nxg - 1) * spacing, (nyg - 1) * spacing
    sides = rng.uniform(side_range[0], side_range[1], n_boxes)
    radii = sides * np.sqrt(3.0) / 2.0
    centers = []
    for b in range(n_boxes):
        for _ in range(100000):
            c = np.array([rng.uniform(radii[b] + 0.5, Lx - radii[b] - 0.5),
                          rng.uniform(radii[b] + 0.5, Ly - radii[b] - 0.5),
                          rng.uniform(radii[b] + 0.1, radii[b] + 2.5)])
            if all(np.linalg.norm(c - centers[k]) > radii[b] + radii[k] + 0.1 for k in range(len(centers))):
                centers.append(c)
                break
        else:
            raise RuntimeError("could not place the boxes")
    parts = []
    for b in range(n_boxes):
        p, n = sample_box(rng, box_pts, sides[b])
        h = np.sqrt(6.0 * sides[b] ** 2 / box_pts)
        R = random_rotation(rng)
        p, n = p @ R.T, n @ R.T
        parts.append((p + centers[b], n, p - 0.6 * h * n + centers[b], centers[b]))
    gx, gy = np.meshgrid(np.arange(nxg) * spacing, np.arange(nyg) * spacing, indexing="ij")
    fp = np.stack([gx.ravel(), gy.ravel(), np.zeros(gx.size)], 1)
    fn = np.tile([0.0, 0.0, 1.0], (fp.shape[0], 1))
    parts.append((fp, fn, fp - 0.6 * spacing * fn, np.array([Lx / 2, Ly / 2, 0.0])))
    areas = [6.0 * s_ ** 2 for s_ in sides] + [nxg * nyg * spacing ** 2]
    return _assemble(f"large{n_boxes}", parts, rho=4.0, lam=1.5, max_super=512, tol=1e-8,
                     meta={"sides": sides, "areas": areas, "static": [n_boxes], "spacing": spacing})


def fibonacci_sphere(npts: int) -> np.ndarray:
    """Quasi-uniform unit vectors (Fibonacci lattice), equal area 4 pi / npts each."""
    i = np.arange(npts) + 0.5
    z = 1.0 - 2.0 * i / npts
    th = np.pi * (1.0 + 5.0 ** 0.5) * i
    r = np.sqrt(1.0 - z * z)
    return np.stack([r * np.cos(th), r * np.sin(th), z], 1)


def ellipsoid_fibonacci_scene(axes, npts: int = 2000, offset: float = 0.15) -> Scene:
    """One ellipsoid at the origin (principal axes along x, y, z) sampled on the
    mapped Fibonacci lattice, with exact quadrature weights
    (4 pi / npts) abc |A^-T u|; sources `offset` inside along the normal.

    A smooth quadrature with the sources more than a point spacing inside:
    its added mass matches Lamb's closed form to ~1e-5 (with random
    area-uniform points and sources closer than the spacing the potential
    between the points is poor and the added mass is off by ~10 %).
    """
    A = np.asarray(axes, dtype=np.float64)
    u = fibonacci_sphere(npts)
    p = u * A
    n = p / (A * A)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    w = (4.0 * np.pi / npts) * np.prod(A) * np.linalg.norm(u / A, axis=1)
    return _assemble(f"ellipsoid_fib{npts}", [(p, n, p - offset * n, np.zeros(3))], rho=3.0, lam=1.5,
                     tol=1e-10, meta={"axes": A[None], "areas": [ellipsoid_area(A)], "weights": w})


def uneven_batch(n_scenes: int = 256, first_seed: int = 3):
    """Scenes of 1-8 ellipsoids with 1500-8000 points per body (seeds 3..258)."""
    out = []
    for k in range(n_scenes):
        rng = np.random.default_rng(first_seed + k)
        nb = int(rng.integers(1, 9))
        counts = rng.integers(1500, 8001, size=nb)
        out.append(ellipsoids_scene(nb, counts, seed=10_000 + first_seed + k))
    return out


def trajectory_poses(n_bodies: int, steps: int, seed: int, dt: float = 0.01, amp_range=(0.05, 0.3)):
    """Smooth rigid motions: each of the 6 DOF of a body is a sum of 4 sinusoids."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(amp_range[0], amp_range[1], size=(n_bodies, 6, 4))
    freq = rng.uniform(0.2, 2.0, size=(n_bodies, 6, 4))
    phase = rng.uniform(0, 2 * np.pi, size=(n_bodies, 6, 4))
    t = np.arange(steps) * dt
    q = (amp[None] * np.sin(2 * np.pi * freq[None] * t[:, None, None, None] + phase[None])).sum(-1)
    v = (amp[None] * 2 * np.pi * freq[None] *
         np.cos(2 * np.pi * freq[None] * t[:, None, None, None] + phase[None])).sum(-1)
    return q, v  # steps x bodies x 6 (translation, rotation vector)


def rotvec_matrix(v) -> np.ndarray:
    """Rotation matrix of a rotation vector (Rodrigues)."""
    v = np.asarray(v, dtype=np.float64)
    th = float(np.linalg.norm(v))
    if th < 1e-300:
        return np.eye(3)
    k = v / th
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    return np.eye(3) + np.sin(th) * K + (1.0 - np.cos(th)) * (K @ K)


def moved(sc: Scene, q) -> Scene:
    """The scene with body b displaced by q[b] = (translation, rotation vector)
    about its centre; points keep their indices (rows, sources, bodies)."""
    q = np.asarray(q, dtype=np.float64)
    x = sc.x.astype(np.float64).copy()
    nx = sc.nx.astype(np.float64).copy()
    y = sc.y.astype(np.float64).copy()
    cen = sc.centers.astype(np.float64).copy()
    for b in range(sc.n_bodies):
        R = rotvec_matrix(q[b, 3:6])
        c = cen[b]
        rows = sc.row_body == b
        srcs = sc.src_body == b
        x[rows] = (x[rows] - c) @ R.T + c + q[b, :3]
        nx[rows] = nx[rows] @ R.T
        y[srcs] = (y[srcs] - c) @ R.T + c + q[b, :3]
        cen[b] = c + q[b, :3]
    nx /= np.linalg.norm(nx, axis=1, keepdims=True)
    meta = dict(sc.meta)
    meta["pose"] = q
    return Scene(name=sc.name, x=_f32(x), nx=_f32(nx), y=_f32(y), row_body=sc.row_body,
                 src_body=sc.src_body, centers=_f32(cen), coef=sc.coef, rho=sc.rho, lam=sc.lam,
                 max_super=sc.max_super, tol=sc.tol, meta=meta)


def trajectory_scene(n_bodies: int = 32, pts: int = 2000, seed: int = 4, steps: int = 500,
                     dt: float = 0.01, amp_range=(0.005, 0.03), box: float = 12.0):
    """The 32-ellipsoid trajectory: a base scene whose bodies are placed with
    room for their motion, and the poses (steps x bodies x 6) and velocities.

    Each DOF is a sum of 4 seeded sinusoids; with amplitudes U(0.005, 0.03)
    a body moves at most 0.12 per axis and turns at most 0.12 rad, and the
    placement margin keeps the bodies apart along the whole trajectory (which
    needs a 12^3 box for 32 bodies).
    """
    rng = np.random.default_rng(seed)
    axes = rng.uniform(0.5, 1.5, size=(n_bodies, 3))
    # a bounding sphere about the centre only translates (by <= sqrt(3) * 4 amp)
    radii = axes.max(axis=1) + np.sqrt(3.0) * 4 * amp_range[1]
    while True:  # grow the box until the seeded placement succeeds
        try:
            centers = random_centers(rng, radii, box)
            break
        except RuntimeError:
            box += 0.5
    parts, rots = [], []
    for b in range(n_bodies):
        p, n = sample_ellipsoid(rng, pts, axes[b])
        R = random_rotation(rng)
        rots.append(R)
        p, n = p @ R.T, n @ R.T
        parts.append((p + centers[b], n, p - 0.05 * n + centers[b], centers[b]))
    base = _assemble(f"trajectory{n_bodies}", parts, rho=3.0, lam=1.5, tol=1e-8,
                     meta={"axes": axes, "areas": [ellipsoid_area(ax) for ax in axes],
                           "rot": np.array(rots)})
    q, v = trajectory_poses(n_bodies, steps, seed + 1, dt, amp_range)
    return base, q, v


def vertex_normals(V, F) -> np.ndarray:
    """Unit vertex normals of a triangle mesh: face normals summed with the
    angle of each face at the vertex as weight."""
    V = np.asarray(V, np.float64)
    p0, p1, p2 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    fn = np.cross(p1 - p0, p2 - p0)
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)

    def angle(a, b):
        c = np.einsum("ij,ij->i", a, b) / (np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1))
        return np.arccos(np.clip(c, -1.0, 1.0))

    ang = [angle(p1 - p0, p2 - p0), angle(p0 - p1, p2 - p1), angle(p0 - p2, p1 - p2)]
    acc = np.zeros_like(V)
    for k in range(3):
        np.add.at(acc, F[:, k], fn * ang[k][:, None])
    return acc / np.linalg.norm(acc, axis=1, keepdims=True)


def mesh_scene(bodies):
    """Triangle-mesh bodies, each (subdivision, semi-axes, rotation vector,
    position, source offset): a scaled, turned icosphere with one source per
    vertex, moved inward along the vertex normal.  Returns a dict of float32
    V, int32 F (global vertex indices), int32 face_body, float32 body_pos,
    float32 S and int32 src_body."""
    Vs, Fs, fb, pos, Ss, sb = [], [], [], [], [], []
    off = 0
    for b, (subdiv, axes, rv, p, depth) in enumerate(bodies):
        V, F = icosphere_mesh(subdiv)
        V = _f32((V * np.asarray(axes, np.float64)) @ rotvec_matrix(rv).T + np.asarray(p, np.float64))
        Ss.append(_f32(V - depth * vertex_normals(V, F)))
        Vs.append(V)
        Fs.append(F + off)
        off += V.shape[0]
        fb.append(np.full(F.shape[0], b, np.int32))
        sb.append(np.full(V.shape[0], b, np.int32))
        pos.append(p)
    return {"V": np.concatenate(Vs).astype(np.float32), "F": np.concatenate(Fs).astype(np.int32),
            "face_body": np.concatenate(fb), "body_pos": _f32(np.array(pos)).astype(np.float32),
            "S": np.concatenate(Ss).astype(np.float32), "src_body": np.concatenate(sb)}
