"""Seeded synthetic point clouds with analytic normals.

The reference is exercised on scanned PLY scenes that are not available here, so
every workload in this package is generated: shapes are sampled uniformly by
surface area with analytic unit normals, placed under known rigid poses, and
surrounded by plane/box clutter.  All randomness flows from one
``numpy.random.Generator`` seeded by the caller, so a (config, seed) pair always
produces the same float32 arrays.

Conventions
-----------
* Clouds are ``(points, normals)`` pairs of ``float32`` arrays of shape ``(n, 3)``.
* A pose ``T`` is a 4x4 ``float64`` matrix mapping model coordinates into scene
  coordinates (``p_scene = R p_model + t``), the same direction as the
  transformation returned by the reference's ``ppf_registration``
  (src/cuda/ppf.cu:74-93).
* The model "diameter" is the maximum axis-aligned extent of the model cloud,
  the rule the reference's driver uses to turn ``tau_d`` into ``d_dist``
  (src/alignment.cpp:246-253).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Cloud",
    "Instance",
    "SceneSpec",
    "uniform_rotation",
    "superellipsoid",
    "torus",
    "capsule_union",
    "spheres_on_slab",
    "box_surface",
    "ground_plane",
    "model_diameter",
    "d_dist_for",
    "transform",
    "config_plain",
    "config_multi_model",
    "config_library",
    "config_large",
    "SYMMETRY",
    "rotation_error_deg",
]


@dataclass
class Cloud:
    points: np.ndarray  # (n, 3) float32
    normals: np.ndarray  # (n, 3) float32

    def __len__(self) -> int:
        return int(self.points.shape[0])

    def subset(self, idx) -> "Cloud":
        return Cloud(self.points[idx].copy(), self.normals[idx].copy())

    @staticmethod
    def concat(clouds) -> "Cloud":
        clouds = list(clouds)
        return Cloud(
            np.concatenate([c.points for c in clouds]).astype(np.float32),
            np.concatenate([c.normals for c in clouds]).astype(np.float32),
        )


@dataclass
class Instance:
    model_index: int
    pose: np.ndarray  # 4x4 float64, model -> scene


@dataclass
class SceneSpec:
    """A generated registration problem: models, one scene, ground truth."""

    models: list
    scene: Cloud
    instances: list
    tau_d: list
    d_dists: list
    diameters: list
    ref_point_df: int = 5
    vote_count_threshold: float = 0.3
    extra: dict = field(default_factory=dict)


# --------------------------------------------------------------------------
# geometry helpers
# --------------------------------------------------------------------------

def _normalize(v):
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    n[n == 0] = 1.0
    return v / n


def uniform_rotation(rng) -> np.ndarray:
    """Uniform random rotation via Shoemake's subgroup algorithm (unit quaternion)."""
    u1, u2, u3 = rng.random(3)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    w = a * np.sin(2 * np.pi * u2)
    x = a * np.cos(2 * np.pi * u2)
    y = b * np.sin(2 * np.pi * u3)
    z = b * np.cos(2 * np.pi * u3)
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
        ]
    )


def make_pose(R, t) -> np.ndarray:
    T = np.eye(4)
    T[:3, :3] = R
    T[:3, 3] = t
    return T


def transform(cloud: Cloud, T) -> Cloud:
    R, t = T[:3, :3], T[:3, 3]
    p = cloud.points.astype(np.float64) @ R.T + t
    n = cloud.normals.astype(np.float64) @ R.T
    return Cloud(p.astype(np.float32), n.astype(np.float32))


def _tilt_normals(rng, normals, degrees):
    """Rotate each normal by ``degrees`` about a random axis perpendicular to it."""
    n = normals.astype(np.float64)
    r = _normalize(rng.normal(size=n.shape))
    perp = _normalize(r - np.sum(r * n, axis=1, keepdims=True) * n)
    ang = np.deg2rad(degrees)
    return _normalize(np.cos(ang) * n + np.sin(ang) * perp)


def add_noise(rng, cloud: Cloud, sigma, tilt_deg) -> Cloud:
    p = cloud.points.astype(np.float64) + rng.normal(scale=sigma, size=cloud.points.shape)
    n = _tilt_normals(rng, cloud.normals, tilt_deg) if tilt_deg > 0 else cloud.normals
    return Cloud(p.astype(np.float32), np.asarray(n, dtype=np.float32))


def model_diameter(cloud: Cloud) -> float:
    """Maximum axis-aligned extent, as computed in float32 by the reference driver."""
    ext = cloud.points.max(axis=0) - cloud.points.min(axis=0)
    return float(np.float32(ext.max()))


def d_dist_for(cloud: Cloud, tau_d: float) -> float:
    return float(np.float32(np.float32(tau_d) * np.float32(model_diameter(cloud))))


def _sample_param_surface(rng, n, f, u_range, v_range, grid=(256, 512)):
    """Sample ``n`` points uniformly by area on a parametric surface.

    ``f(u, v) -> (points, normals)``.  The parameter domain is cut into a grid of
    cells; a cell is chosen with probability proportional to its (numerically
    estimated) area and a parameter is drawn uniformly inside it, so the
    sampling is area-uniform up to the grid resolution and every sample lies
    exactly on the surface.
    """
    gu, gv = grid
    u0, u1 = u_range
    v0, v1 = v_range
    ue = np.linspace(u0, u1, gu + 1)
    ve = np.linspace(v0, v1, gv + 1)
    uc = 0.5 * (ue[:-1] + ue[1:])
    vc = 0.5 * (ve[:-1] + ve[1:])
    U, V = np.meshgrid(uc, vc, indexing="ij")
    du = (u1 - u0) / gu
    dv = (v1 - v0) / gv
    # area of each cell from its four corners (two triangles)
    Ue, Ve = np.meshgrid(ue, ve, indexing="ij")
    P, _ = f(Ue.ravel(), Ve.ravel())
    P = P.reshape(gu + 1, gv + 1, 3)
    a = P[:-1, :-1]
    b = P[1:, :-1]
    c = P[1:, 1:]
    d = P[:-1, 1:]
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=-1) + 0.5 * np.linalg.norm(
        np.cross(c - a, d - a), axis=-1
    )
    p = area.ravel() / area.sum()
    cells = rng.choice(p.size, size=n, p=p)
    uu = U.ravel()[cells] + (rng.random(n) - 0.5) * du
    vv = V.ravel()[cells] + (rng.random(n) - 0.5) * dv
    pts, nrm = f(uu, vv)
    return pts, _normalize(nrm)


def _spow(x, e):
    return np.sign(x) * np.abs(x) ** e


def superellipsoid(rng, n, axes=(0.10, 0.06, 0.04), e1=0.5, e2=1.0) -> Cloud:
    """Barr superellipsoid: x = a C(eta)^e1 C(w)^e2, y = b C(eta)^e1 S(w)^e2, z = c S(eta)^e1."""
    a, b, c = axes

    def f(eta, w):
        ce, se = np.cos(eta), np.sin(eta)
        cw, sw = np.cos(w), np.sin(w)
        pts = np.stack(
            [a * _spow(ce, e1) * _spow(cw, e2), b * _spow(ce, e1) * _spow(sw, e2), c * _spow(se, e1)],
            axis=-1,
        )
        nrm = np.stack(
            [
                _spow(ce, 2 - e1) * _spow(cw, 2 - e2) / a,
                _spow(ce, 2 - e1) * _spow(sw, 2 - e2) / b,
                _spow(se, 2 - e1) / c,
            ],
            axis=-1,
        )
        return pts, nrm

    pts, nrm = _sample_param_surface(rng, n, f, (-np.pi / 2, np.pi / 2), (-np.pi, np.pi))
    return Cloud(pts.astype(np.float32), nrm.astype(np.float32))


def torus(rng, n, R=0.08, r=0.025) -> Cloud:
    def f(u, v):
        pts = np.stack([(R + r * np.cos(v)) * np.cos(u), (R + r * np.cos(v)) * np.sin(u), r * np.sin(v)], -1)
        nrm = np.stack([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)], -1)
        return pts, nrm

    pts, nrm = _sample_param_surface(rng, n, f, (0, 2 * np.pi), (0, 2 * np.pi))
    return Cloud(pts.astype(np.float32), nrm.astype(np.float32))


def _capsule_samples(rng, m, A, B, rad):
    """Uniform samples on a capsule surface (cylinder + two hemispheres)."""
    axis = B - A
    L = np.linalg.norm(axis)
    ax = axis / L
    tmp = np.array([1.0, 0, 0]) if abs(ax[0]) < 0.9 else np.array([0, 1.0, 0])
    e1 = _normalize(np.cross(ax, tmp))
    e2 = np.cross(ax, e1)
    cyl_area = 2 * np.pi * rad * L
    sph_area = 4 * np.pi * rad * rad
    k_cyl = rng.binomial(m, cyl_area / (cyl_area + sph_area))
    t = rng.random(k_cyl) * L
    th = rng.random(k_cyl) * 2 * np.pi
    nc = np.cos(th)[:, None] * e1 + np.sin(th)[:, None] * e2
    pc = A + t[:, None] * ax + rad * nc
    k_s = m - k_cyl
    d = _normalize(rng.normal(size=(k_s, 3)))
    end = np.where((d @ ax)[:, None] > 0, B, A)
    ps = end + rad * d
    return np.concatenate([pc, ps]), np.concatenate([nc, d])


def _dist_to_segment(p, A, B):
    ab = B - A
    t = np.clip(((p - A) @ ab) / (ab @ ab), 0, 1)
    return np.linalg.norm(p - (A + t[:, None] * ab), axis=1)


def capsule_union(rng, n) -> Cloud:
    """Union of three random capsules that share a common core region."""
    caps = []
    for _ in range(3):
        d = _normalize(rng.normal(size=3))
        L = rng.uniform(0.07, 0.13)
        c = rng.uniform(-0.015, 0.015, size=3)
        rad = rng.uniform(0.015, 0.028)
        caps.append((c - 0.5 * L * d, c + 0.5 * L * d, rad))
    areas = np.array([2 * np.pi * r * np.linalg.norm(B - A) + 4 * np.pi * r * r for A, B, r in caps])
    pts_all, nrm_all = [], []
    have = 0
    while have < n:
        m = int((n - have) * 1.6) + 64
        per = rng.multinomial(m, areas / areas.sum())
        for ci, (A, B, rad) in enumerate(caps):
            p, q = _capsule_samples(rng, per[ci], A, B, rad)
            keep = np.ones(len(p), bool)
            for cj, (A2, B2, r2) in enumerate(caps):
                if cj != ci:
                    keep &= _dist_to_segment(p, A2, B2) > r2
            pts_all.append(p[keep])
            nrm_all.append(q[keep])
            have += int(keep.sum())
    p = np.concatenate(pts_all)
    q = np.concatenate(nrm_all)
    sel = rng.permutation(len(p))[:n]
    return Cloud(p[sel].astype(np.float32), q[sel].astype(np.float32))


def box_surface(rng, n, lo, hi, faces=6) -> Cloud:
    """Uniform samples on an axis-aligned box surface (6 faces, or 5 without the bottom)."""
    lo = np.asarray(lo, float)
    hi = np.asarray(hi, float)
    s = hi - lo
    face_defs = []  # (axis, side)
    for axis in range(3):
        for side in (0, 1):
            if faces == 5 and axis == 2 and side == 0:
                continue
            face_defs.append((axis, side))
    areas = np.array([np.prod(np.delete(s, ax)) for ax, _ in face_defs])
    per = rng.multinomial(n, areas / areas.sum())
    pts, nrm = [], []
    for (ax, side), k in zip(face_defs, per):
        p = lo + rng.random((k, 3)) * s
        p[:, ax] = hi[ax] if side else lo[ax]
        q = np.zeros((k, 3))
        q[:, ax] = 1.0 if side else -1.0
        pts.append(p)
        nrm.append(q)
    return Cloud(np.concatenate(pts).astype(np.float32), np.concatenate(nrm).astype(np.float32))


def spheres_on_slab(rng, n, rows=2, cols=3) -> Cloud:
    """A slab with a rows x cols grid of random-radius spheres sunk partly into its top face."""
    sx, sy, sz = 0.18, 0.12, 0.02
    lo = np.array([-sx / 2, -sy / 2, -sz / 2])
    hi = -lo
    spheres = []
    for i in range(rows):
        for j in range(cols):
            rad = rng.uniform(0.012, 0.022)
            cx = lo[0] + (j + 0.5) * sx / cols
            cy = lo[1] + (i + 0.5) * sy / rows
            spheres.append((np.array([cx, cy, hi[2] + 0.5 * rad]), rad))
    slab_area = 2 * (sx * sy + sx * sz + sy * sz)
    sph_area = sum(4 * np.pi * r * r for _, r in spheres)
    pts_all, nrm_all = [], []
    have = 0
    while have < n:
        m = int((n - have) * 1.5) + 64
        k_slab = rng.binomial(m, slab_area / (slab_area + sph_area))
        b = box_surface(rng, k_slab, lo, hi)
        p = b.points.astype(float)
        q = b.normals.astype(float)
        keep = np.ones(len(p), bool)
        for c, r in spheres:
            keep &= np.linalg.norm(p - c, axis=1) > r
        pts_all.append(p[keep])
        nrm_all.append(q[keep])
        have += int(keep.sum())
        k_s = m - k_slab
        radii = np.array([r for _, r in spheres])
        per = rng.multinomial(k_s, radii**2 / np.sum(radii**2))
        for (c, r), k in zip(spheres, per):
            d = _normalize(rng.normal(size=(k, 3)))
            p = c + r * d
            keep = ~np.all((p >= lo) & (p <= hi), axis=1)
            pts_all.append(p[keep])
            nrm_all.append(d[keep])
            have += int(keep.sum())
    p = np.concatenate(pts_all)
    q = np.concatenate(nrm_all)
    sel = rng.permutation(len(p))[:n]
    return Cloud(p[sel].astype(np.float32), q[sel].astype(np.float32))


def ground_plane(rng, n, z, half_extent, center=(0.0, 0.0)) -> Cloud:
    p = np.empty((n, 3))
    p[:, 0] = center[0] + rng.uniform(-half_extent, half_extent, n)
    p[:, 1] = center[1] + rng.uniform(-half_extent, half_extent, n)
    p[:, 2] = z
    q = np.zeros((n, 3))
    q[:, 2] = 1.0
    return Cloud(p.astype(np.float32), q.astype(np.float32))


def occlude(rng, cloud: Cloud, fraction) -> Cloud:
    """Delete ``fraction`` of the points lying on one side of a random plane.

    The plane's normal is uniform on the sphere and it is offset from the
    cloud's centroid to the quantile that removes exactly ``fraction`` of the
    points (a plane through the centroid itself would remove about half).
    """
    if fraction <= 0:
        return cloud
    d = _normalize(rng.normal(size=3))
    s = (cloud.points.astype(np.float64) - cloud.points.mean(axis=0)) @ d
    thr = np.quantile(s, 1.0 - fraction)
    keep = s <= thr
    return cloud.subset(np.nonzero(keep)[0])


SHAPES = ("superellipsoid", "torus", "capsules", "spheres_slab")


def _rot(axis, angle):
    c, s_ = np.cos(angle), np.sin(angle)
    if axis == "x":
        return np.array([[1, 0, 0], [0, c, -s_], [0, s_, c]])
    if axis == "y":
        return np.array([[c, 0, s_], [0, 1, 0], [-s_, 0, c]])
    return np.array([[c, -s_, 0], [s_, c, 0], [0, 0, 1]])


# Rotations (in the model's own frame) that map each shape family onto
# itself: the superellipsoid's three half-turns, the spheres-on-slab grid's
# half-turn about z (exact for the slab and the sphere centres; the sphere
# radii differ, so only approximately for the surface); the torus is
# symmetric under every rotation about z and a half-turn about x ("axis");
# the capsule union has none.
SYMMETRY = {
    "superellipsoid": [np.eye(3), _rot("x", np.pi), _rot("y", np.pi), _rot("z", np.pi)],
    "torus": "axis",
    "capsules": [np.eye(3)],
    "spheres_slab": [np.eye(3), _rot("z", np.pi)],
}


def rotation_error_deg(R, G, family=None):
    """Angle in degrees between rotations R and G, or with a shape family the
    smallest angle over the rotations its symmetry makes equivalent."""
    R = np.asarray(R, np.float64)
    G = np.asarray(G, np.float64)

    def ang(A, B):
        return float(np.degrees(np.arccos(np.clip((np.trace(A.T @ B) - 1) / 2, -1, 1))))

    sym = SYMMETRY.get(family, [np.eye(3)]) if family else [np.eye(3)]
    if isinstance(sym, str):  # axis symmetry about the model's z
        c = float(np.clip(abs((R[:, 2]) @ G[:, 2]), -1, 1))
        return float(np.degrees(np.arccos(c)))
    return min(ang(R @ S, G) for S in sym)


def make_shape(rng, family, n) -> Cloud:
    if family == "superellipsoid":
        return superellipsoid(rng, n)
    if family == "torus":
        return torus(rng, n)
    if family == "capsules":
        return capsule_union(rng, n)
    if family == "spheres_slab":
        return spheres_on_slab(rng, n)
    raise ValueError(family)


def _place_scene(rng, models, model_ids, n_scene, occlusion, sigma, tilt_deg, n_boxes,
                 spacing=0.32, plane_fraction=0.6):
    """Place model instances on a jittered grid above a ground plane, add box clutter."""
    k = len(model_ids)
    cols = int(np.ceil(np.sqrt(k)))
    parts, instances = [], []
    for slot, mi in enumerate(model_ids):
        R = uniform_rotation(rng)
        gx, gy = slot % cols, slot // cols
        t = np.array(
            [
                (gx - 0.5 * (cols - 1)) * spacing + rng.uniform(-0.03, 0.03),
                (gy - 0.5 * (cols - 1)) * spacing + rng.uniform(-0.03, 0.03),
                rng.uniform(0.0, 0.05),
            ]
        )
        T = make_pose(R, t)
        inst = transform(models[mi], T)
        inst = occlude(rng, inst, occlusion)
        parts.append(inst)
        instances.append(Instance(mi, T))
    n_obj = sum(len(p) for p in parts)
    n_clutter = max(n_scene - n_obj, 0)
    half = 0.5 * spacing * cols + 0.15
    n_plane = int(round(n_clutter * plane_fraction))
    n_box = n_clutter - n_plane
    parts.append(ground_plane(rng, n_plane, -0.16, half))
    if n_boxes > 0 and n_box > 0:
        per = rng.multinomial(n_box, np.ones(n_boxes) / n_boxes)
        for b in range(n_boxes):
            side = rng.uniform(0.05, 0.12, size=3)
            cxy = rng.uniform(-half + 0.08, half - 0.08, size=2)
            lo = np.array([cxy[0] - side[0] / 2, cxy[1] - side[1] / 2, -0.16])
            parts.append(box_surface(rng, per[b], lo, lo + side, faces=5))
    scene = Cloud.concat(parts)
    scene = add_noise(rng, scene, sigma, tilt_deg)
    return scene, instances


def config_plain(seed=1000, n_model=2000, n_plane=6000, n_box=2000, sigma=5e-4, tilt_deg=2.0,
                 tau_d=0.05, ref_point_df=5, vote_count_threshold=0.3) -> SceneSpec:
    """One model, one scene: superellipsoid (semi-axes 0.10/0.06/0.04 m, e1=0.5, e2=1.0),
    the scene holding that model under a uniform random rotation and a translation
    uniform in [-0.15, 0.15]^3 m, plus a ground plane and two axis-aligned boxes."""
    rng = np.random.default_rng(seed)
    model = superellipsoid(rng, n_model)
    R = uniform_rotation(rng)
    t = rng.uniform(-0.15, 0.15, size=3)
    T = make_pose(R, t)
    obj = transform(model, T)
    plane = ground_plane(rng, n_plane, -0.3, 0.35)
    boxes = []
    per = rng.multinomial(n_box, [0.5, 0.5])
    for b in range(2):
        side = rng.uniform(0.05, 0.12, size=3)
        cxy = rng.uniform(-0.25, 0.25, size=2)
        lo = np.array([cxy[0] - side[0] / 2, cxy[1] - side[1] / 2, -0.3])
        boxes.append(box_surface(rng, per[b], lo, lo + side, faces=5))
    scene = add_noise(rng, Cloud.concat([obj, plane] + boxes), sigma, tilt_deg)
    diam = model_diameter(model)
    return SceneSpec(
        models=[model],
        scene=scene,
        instances=[Instance(0, T)],
        tau_d=[tau_d],
        d_dists=[d_dist_for(model, tau_d)],
        diameters=[diam],
        ref_point_df=ref_point_df,
        vote_count_threshold=vote_count_threshold,
    )


def config_multi_model(seed=1001, n_scene=60000, occlusion=0.3, sigma=5e-4, tilt_deg=0.0,
                       tau_d=(0.03, 0.035, 0.03, 0.05), ref_point_df=5,
                       vote_count_threshold=0.3, sizes=None) -> SceneSpec:
    """Four models (superellipsoid, torus, 3-capsule union, 2x3 spheres on a slab) of
    3k-6k points each, all placed in one 60k-point scene, each 30% occluded, with a
    ground plane and five boxes as clutter."""
    rng = np.random.default_rng(seed)
    if sizes is None:
        sizes = [int(s) for s in rng.integers(3000, 6001, size=4)]
    models = [make_shape(rng, fam, n) for fam, n in zip(SHAPES, sizes)]
    scene, inst = _place_scene(rng, models, [0, 1, 2, 3], n_scene, occlusion, sigma, tilt_deg, 5)
    return SceneSpec(
        models=models,
        scene=scene,
        instances=inst,
        tau_d=list(tau_d),
        d_dists=[d_dist_for(m, td) for m, td in zip(models, tau_d)],
        diameters=[model_diameter(m) for m in models],
        ref_point_df=ref_point_df,
        vote_count_threshold=vote_count_threshold,
        extra={"families": list(SHAPES)},
    )


def config_library(seed=1002, n_models=16, n_scenes=256, model_range=(2000, 20000),
                   scene_range=(5000, 200000), occlusion=0.3, sigma=5e-4, tau_d=0.04):
    """A model library (shape families cycled, sizes log-uniform) and scenes of
    log-uniform sizes, each holding 1-4 library models.  Returns
    ``(models, d_dists, scenes)`` with ``scenes`` a list of ``(Cloud, [Instance])``."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(model_range[0]), np.log(model_range[1])
    sizes = np.exp(rng.uniform(lo, hi, n_models)).astype(int)
    models = [make_shape(rng, SHAPES[i % 4], int(s)) for i, s in enumerate(sizes)]
    d_dists = [d_dist_for(m, tau_d) for m in models]
    scenes = []
    slo, shi = np.log(scene_range[0]), np.log(scene_range[1])
    for _ in range(n_scenes):
        ns = int(np.exp(rng.uniform(slo, shi)))
        k = int(rng.integers(1, 5))
        ids = [int(x) for x in rng.choice(n_models, size=k, replace=False)]
        sc, inst = _place_scene(rng, models, ids, ns, occlusion, sigma, 0.0, 5)
        scenes.append((sc, inst))
    return models, d_dists, scenes


def config_large(seed=1004, n_model=40000, n_scene=1_000_000, instances=10, occlusion=0.4,
                 sigma=1e-3, tau_d=0.025):
    """Dense superquadric + torus union model, a 1M-point scene with 10 instances."""
    rng = np.random.default_rng(seed)
    a = superellipsoid(rng, n_model // 2)
    b = transform(torus(rng, n_model - n_model // 2), make_pose(np.eye(3), [0.0, 0.0, 0.05]))
    model = Cloud.concat([a, b])
    scene, inst = _place_scene(rng, [model], [0] * instances, n_scene, occlusion, sigma, 0.0, 12,
                               spacing=0.35)
    return SceneSpec(
        models=[model],
        scene=scene,
        instances=inst,
        tau_d=[tau_d],
        d_dists=[d_dist_for(model, tau_d)],
        diameters=[model_diameter(model)],
        ref_point_df=5,
    )
