"""Seeded synthetic scenes standing in for the reference's benchmark scenes.

The reference measures whole frames of its demo scenes through WebGPU (examples/demo/ruinsScene.ts,
worldScene.ts, stressScene.ts; numbers in docs/benchmarks.json). Those need a browser and a graphics API, so the
workloads here are seeded synthetic scenes with the published shapes and sizes:

* ``plain_small``: one displaced icosphere (20 n^2 triangles, n = 229 -> 1,048,820, the icosphere count nearest
  to 1,048,576), 64 instances on an 8 x 8 grid 3 radii apart, yaw U[0, 2 pi), scale lognormal(0, 0.25), one
  1920 x 1080 camera outside the grid looking at its centre; threshold 1 px, frustum + size culling.
* ``ruins``: 40 meshes of 50k-2M triangles (log-uniform; displaced icospheres and box lattices), 113,106 instances
  uniform over 1 km x 1 km, yaw U[0, 2 pi), scale lognormal(0, 0.3); mesh choice weighted by 1 / triangles so the
  full-detail total lands near the reference ruins scene's 5.73 billion triangles (docs/benchmarks.json);
  1080p camera on a seeded 32-pose spline at 2 m height; HZB from a 1920 x 1080 depth image of 64 screen-aligned
  occluder quads at U[5, 500] m.
* ``large_world``: 3,000,000 instances of the same 40 meshes over 6 km x 6 km, 80% on a jittered grid (blue noise
  with a guaranteed minimum spacing, standing in for Poisson-disk placement) and 20% in 50 seeded towns of 150 m
  radius; 16 poses of a 3840 x 2160 camera at 2 m height; triangleBudget 6,000,000; maxDrawDistance 400 m on the
  bucket of small meshes (the 10 with the fewest triangles: none of the 50k-2M meshes is under 10k triangles).
* ``serving_scenes``: 16 scenes of 10k-3M instances (log-uniform) of the same meshes at the ruins density, and a
  seeded request stream over them (pose, resolution 720p / 1080p / 4K, threshold U[0.5, 2], budget on a quarter).

Instance fields of the large scenes come from numpy's seeded PCG64 stream (vectorised; millions of instances).
"""
from __future__ import annotations

import math
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import build as B
from .camera import Camera, compose, look_at_world, invert_rigid, perspective


def rng_normal(r: B.Mulberry32) -> float:
    """Standard normal from the seeded stream (Box-Muller)."""
    u1 = max(r(), 1e-12)
    u2 = r()
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(2 * math.pi * u2)


@dataclass
class SceneSpec:
    name: str
    meshes: list = field(default_factory=list)          # VirtualMeshData per mesh
    mesh_triangles: list = field(default_factory=list)  # leaf triangles per mesh
    instances: list = field(default_factory=list)       # (n_i, 16) float32 matrices per mesh
    cameras: list = field(default_factory=list)
    depth_images: list = field(default_factory=list)    # per camera (or empty)
    notes: dict = field(default_factory=dict)

    @property
    def instance_count(self) -> int:
        return int(sum(len(m) for m in self.instances))

    @property
    def full_detail_triangles(self) -> int:
        return int(sum(len(m) * t for m, t in zip(self.instances, self.mesh_triangles)))


def icosphere_mesh(n: int, radius: float = 1.0, amplitude: float = 0.02, seed: int = 1, threads: int = 0):
    pos, idx = B.gen_icosphere(n, radius, amplitude, 3.0, seed)
    return B.build_virtual_mesh(pos, idx, threads=threads)


def plain_small(n: int = 229, seed: int = 1, grid: int = 8, threads: int = 0) -> SceneSpec:
    """The small plain scene of the module docstring; `n` may be lowered for CPU-sized tests."""
    r = B.Mulberry32(seed)
    R = 1.0
    data = icosphere_mesh(n, R, 0.02, seed, threads)
    mats = []
    spacing = 3 * R
    for iz in range(grid):
        for ix in range(grid):
            yaw = r() * 2 * math.pi
            s = math.exp(0.25 * rng_normal(r))
            x = (ix - (grid - 1) / 2) * spacing
            z = (iz - (grid - 1) / 2) * spacing
            mats.append(compose((x, 0.0, z), yaw, s))
    half = grid * spacing / 2
    ang = r() * 2 * math.pi
    dist = half * (1.6 + r())
    eye = (math.cos(ang) * dist, half * (0.3 + 0.5 * r()), math.sin(ang) * dist)
    cam = Camera.perspective_look_at(eye, (0, 0, 0), 60.0, 1920, 1080, 0.1, 1000.0)
    spec = SceneSpec("plain_small", [data], [data.stats["leafTriangles"]], [np.array(mats, np.float32)], [cam])
    spec.notes = dict(triangles=20 * n * n, grid=grid, spacing=spacing)
    return spec


def _ruins_meshes(count: int, tri_lo: float, tri_hi: float, seed: int, threads: int):
    r = B.Mulberry32(seed * 7919 + 13)
    jobs = []
    for i in range(count):
        # stratified log-uniform: one draw per equal log-width stratum, so the smallest mesh is near tri_lo
        tris = math.exp(math.log(tri_lo) + (i + r()) / count * (math.log(tri_hi) - math.log(tri_lo)))
        if i % 2 == 0:  # displaced icosphere (rocks, boulders)
            n = max(2, int(round(math.sqrt(tris / 20))))
            radius = 1.0 + 3.0 * r()
            jobs.append(("ico", n, radius, 0.04 + 0.06 * r(), seed * 100 + i))
        else:  # box lattice (walls, pillars, blocks)
            boxes = 4 + int(r() * 12)
            k = max(1, int(round(math.sqrt(tris / (12 * boxes)))))
            jobs.append(("box", boxes, k, 2.0 + 4.0 * r(), seed * 100 + i))

    def make(job):
        if job[0] == "ico":
            _, n, radius, amp, s = job
            pos, idx = B.gen_icosphere(n, radius, amp, 2.5, s)
        else:
            _, boxes, k, extent, s = job
            pos, idx = B.gen_box_lattice(boxes, k, extent, s)
        return B.build_virtual_mesh(pos, idx, threads=1)

    with ThreadPoolExecutor(max_workers=threads or None) as ex:
        return list(ex.map(make, jobs))


def ruins(seed: int = 2, mesh_count: int = 40, tri_lo: float = 50_000, tri_hi: float = 2_000_000,
          instances: int = 113_106, extent: float = 1000.0, poses: int = 32, width: int = 1920, height: int = 1080,
          target_full_detail: float = 5.73e9, quads: int = 64, threads: int = 0) -> SceneSpec:
    """The ruins-like scene of the module docstring. Smaller arguments give CPU-sized variants for tests."""
    meshes = _ruins_meshes(mesh_count, tri_lo, tri_hi, seed, threads)
    tris = np.array([m.stats["leafTriangles"] for m in meshes], np.float64)
    # weights ~ tris^-a; pick a so the expected full-detail total is near the target
    best = None
    for a in np.linspace(0.0, 12.0, 1201):
        w = tris ** (-a)
        w /= w.sum()
        total = instances * float((w * tris).sum())
        if best is None or abs(math.log(total / target_full_detail)) < abs(math.log(best[1] / target_full_detail)):
            best = (a, total, w)
    a, _, w = best
    r = B.Mulberry32(seed)
    counts = np.zeros(mesh_count, np.int64)
    cdf = np.cumsum(w)
    choice = np.empty(instances, np.int64)
    xs = np.empty(instances)
    zs = np.empty(instances)
    yaws = np.empty(instances)
    scales = np.empty(instances)
    for i in range(instances):
        choice[i] = min(int(np.searchsorted(cdf, r())), mesh_count - 1)
        xs[i] = (r() - 0.5) * extent
        zs[i] = (r() - 0.5) * extent
        yaws[i] = r() * 2 * math.pi
        scales[i] = math.exp(0.3 * rng_normal(r))
    per_mesh = []
    for m in range(mesh_count):
        sel = np.nonzero(choice == m)[0]
        counts[m] = len(sel)
        c, s = np.cos(yaws[sel]), np.sin(yaws[sel])
        mat = np.zeros((len(sel), 16), np.float32)
        mat[:, 0], mat[:, 2] = c * scales[sel], -s * scales[sel]
        mat[:, 5] = scales[sel]
        mat[:, 8], mat[:, 10] = s * scales[sel], c * scales[sel]
        mat[:, 12], mat[:, 13], mat[:, 14], mat[:, 15] = xs[sel], 0.0, zs[sel], 1.0
        per_mesh.append(mat)
    # camera spline at 2 m height: Catmull-Rom through seeded control points inside the square
    ctrl = [((r() - 0.5) * extent * 0.8, (r() - 0.5) * extent * 0.8) for _ in range(8)]
    cams = []
    depth = []
    near, far = 0.1, 5000.0
    proj = perspective(60.0, width / height, near, far)
    for k in range(poses):
        t = k / poses * (len(ctrl) - 3)
        i = int(t)
        f = t - i
        p0, p1, p2, p3 = ctrl[i], ctrl[i + 1], ctrl[i + 2], ctrl[i + 3]

        def cr(a0, a1, a2, a3, u):
            return 0.5 * ((2 * a1) + (-a0 + a2) * u + (2 * a0 - 5 * a1 + 4 * a2 - a3) * u * u +
                          (-a0 + 3 * a1 - 3 * a2 + a3) * u ** 3)

        x = cr(p0[0], p1[0], p2[0], p3[0], f)
        z = cr(p0[1], p1[1], p2[1], p3[1], f)
        x2 = cr(p0[0], p1[0], p2[0], p3[0], min(f + 0.05, 1.0))
        z2 = cr(p0[1], p1[1], p2[1], p3[1], min(f + 0.05, 1.0))
        dx, dz = x2 - x, z2 - z
        if dx * dx + dz * dz < 1e-9:
            dx, dz = 1.0, 0.0
        eye = (x, 2.0, z)
        target = (x + dx, 2.0 - 0.02 * math.hypot(dx, dz), z + dz)
        world = look_at_world(eye, target)
        cams.append(Camera(view=invert_rigid(world), proj=proj.copy(), near=near, height=float(height),
                           width=float(width), extra={"eye": np.array(eye)}))
        if quads:
            depth.append(B.gen_depth_image(width, height, quads, 5.0, 500.0, float(proj[10]), float(proj[14]),
                                           seed * 1000 + k))
    spec = SceneSpec("ruins", meshes, [int(t) for t in tris], per_mesh, cams, depth)
    spec.notes = dict(weight_exponent=float(a), expected_full_detail=float(best[1]),
                      mesh_counts=counts.tolist(), meshlets=int(sum(m.meshlet_count for m in meshes)))
    return spec


def load_into(vg, spec: SceneSpec, **mesh_options) -> list:
    """Creates every mesh of `spec` in a VirtualGeometry context (slot order = mesh order)."""
    out = []
    for data, mats in zip(spec.meshes, spec.instances):
        out.append(vg.create_mesh(data, mats, **mesh_options))
    return out


def batching_views(ruins: SceneSpec, cameras: int = 64, seed: int = 21) -> list:
    """The batching workload over the ruins-like scene: `cameras` cameras at the spline's eye points with seeded yaw,
    resolutions cycling 1280x720 / 1920x1080 / 3840x2160 and thresholds 0.5 / 1 / 2 px, each followed by its 4
    orthographic shadow cascades (splits 0.1-10-40-150-600 m, light direction (0.35, -1, 0.25)). Returns
    (camera, lever dict) per view in launch order: camera, then its cascades; the dict holds error_threshold and,
    for a cascade, cascade_clip (a camera view has no shadow sweep)."""
    from .camera import cascade_clips
    rng = np.random.default_rng(seed)
    sizes = [(1280, 720), (1920, 1080), (3840, 2160)]
    thresholds = [0.5, 1.0, 2.0]
    light = (0.35, -1.0, 0.25)
    out = []
    for i in range(cameras):
        eye = ruins.cameras[i % len(ruins.cameras)].extra["eye"]
        yaw = rng.uniform(0, 2 * np.pi)
        w, h = sizes[i % 3]
        t = thresholds[(i // 3) % 3]
        cam = Camera.perspective_look_at(tuple(eye), (eye[0] + np.cos(yaw), eye[1] - 0.02, eye[2] + np.sin(yaw)), 60,
                                         w, h, 0.1, 5000.0)
        out.append((cam, dict(error_threshold=t)))
        for clip in cascade_clips(cam, light, [0.1, 10.0, 40.0, 150.0, 600.0]):
            out.append((cam, dict(error_threshold=t, cascade_clip=clip)))
    return out


# ---------------------------------------------------------------------------------------------------- large scenes
def _weights(tris: np.ndarray, exponent: float) -> np.ndarray:
    w = tris.astype(np.float64) ** (-exponent)
    return w / w.sum()


def _matrices(rng: np.random.Generator, xs: np.ndarray, zs: np.ndarray, scale_sigma: float) -> np.ndarray:
    n = len(xs)
    yaw = rng.uniform(0.0, 2 * math.pi, n)
    sc = np.exp(scale_sigma * rng.standard_normal(n))
    c, s = np.cos(yaw), np.sin(yaw)
    mat = np.zeros((n, 16), np.float32)
    mat[:, 0], mat[:, 2] = c * sc, -s * sc
    mat[:, 5] = sc
    mat[:, 8], mat[:, 10] = s * sc, c * sc
    mat[:, 12], mat[:, 14], mat[:, 15] = xs, zs, 1.0
    return mat


def _jittered_grid(rng: np.random.Generator, n: int, extent: float) -> tuple[np.ndarray, np.ndarray]:
    """n points on distinct cells of a square grid over [-extent/2, extent/2]^2, each jittered inside the middle
    70% of its cell: blue noise whose points are at least 0.3 cell apart."""
    g = int(math.ceil(math.sqrt(n * 1.25)))
    cells = rng.choice(g * g, n, replace=False)
    size = extent / g
    cx, cz = cells % g, cells // g
    xs = (cx + 0.5 + rng.uniform(-0.35, 0.35, n)) * size - extent / 2
    zs = (cz + 0.5 + rng.uniform(-0.35, 0.35, n)) * size - extent / 2
    return xs, zs


def _ground_cameras(rng: np.random.Generator, n: int, extent: float, sizes, near=0.1, far=10000.0) -> list:
    cams = []
    for _ in range(n):
        x, z = rng.uniform(-0.45, 0.45, 2) * extent
        yaw = rng.uniform(0.0, 2 * math.pi)
        width, height = sizes[int(rng.integers(len(sizes)))]
        eye = (float(x), 2.0, float(z))
        target = (float(x + math.cos(yaw)), 2.0 - 0.02, float(z + math.sin(yaw)))
        cams.append(Camera(view=invert_rigid(look_at_world(eye, target)), proj=perspective(60.0, width / height, near, far),
                           near=near, height=float(height), width=float(width), extra={"eye": np.array(eye)}))
    return cams


def _assign(rng: np.random.Generator, weights: np.ndarray, xs, zs, scale_sigma: float) -> list:
    choice = rng.choice(len(weights), len(xs), p=weights)
    mats = _matrices(rng, xs, zs, scale_sigma)
    return [mats[choice == m] for m in range(len(weights))]


def large_world(meshes: list, mesh_triangles: list, weight_exponent: float, seed: int = 5, instances: int = 3_000_000,
                extent: float = 6000.0, towns: int = 50, town_fraction: float = 0.2, town_radius: float = 150.0,
                poses: int = 16, width: int = 3840, height: int = 2160) -> SceneSpec:
    """The large-world scene of the module docstring over already built meshes."""
    rng = np.random.default_rng(seed)
    n_town = int(instances * town_fraction)
    xs, zs = _jittered_grid(rng, instances - n_town, extent)
    centres = rng.uniform(-0.45, 0.45, (towns, 2)) * extent
    which = rng.integers(towns, size=n_town)
    r = town_radius * np.sqrt(rng.uniform(0.0, 1.0, n_town))
    a = rng.uniform(0.0, 2 * math.pi, n_town)
    xs = np.concatenate([xs, centres[which, 0] + r * np.cos(a)])
    zs = np.concatenate([zs, centres[which, 1] + r * np.sin(a)])
    tris = np.asarray(mesh_triangles, np.float64)
    per_mesh = _assign(rng, _weights(tris, weight_exponent), xs, zs, 0.3)
    cams = _ground_cameras(rng, poses, extent, [(width, height)])
    small = [int(i) for i in np.argsort(tris)[:10]]
    spec = SceneSpec("large_world", meshes, [int(t) for t in tris], per_mesh, cams, [])
    spec.notes = dict(small_meshes=small, max_draw_distance=400.0, triangle_budget=6_000_000.0,
                      placement="jittered grid (min spacing 0.3 cell) + 50 towns", seed=seed)
    return spec


def serving_scenes(meshes: list, mesh_triangles: list, weight_exponent: float, seed: int = 9, count: int = 16,
                   lo: int = 10_000, hi: int = 3_000_000, density_per_km2: float = 113_106.0) -> list:
    """`count` scenes of log-uniform instance counts in [lo, hi] at the ruins density (list of SceneSpec)."""
    rng = np.random.default_rng(seed)
    tris = np.asarray(mesh_triangles, np.float64)
    w = _weights(tris, weight_exponent)
    out = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        extent = 1000.0 * math.sqrt(n / density_per_km2)
        xs = rng.uniform(-0.5, 0.5, n) * extent
        zs = rng.uniform(-0.5, 0.5, n) * extent
        spec = SceneSpec(f"serve{k}", meshes, [int(t) for t in tris], _assign(rng, w, xs, zs, 0.3), [], [])
        spec.notes = dict(extent=extent)
        out.append(spec)
    return out


def request_stream(specs: list, count: int, rate_per_s: float, seed: int = 13, budget_fraction: float = 0.25) -> list:
    """Seeded requests over `specs`: (arrival seconds (Poisson process), scene index, camera, threshold, budget)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, count))
    out = []
    sizes = [(1280, 720), (1920, 1080), (3840, 2160)]
    for i in range(count):
        k = int(rng.integers(len(specs)))
        cam = _ground_cameras(rng, 1, specs[k].notes["extent"], sizes)[0]
        threshold = float(rng.uniform(0.5, 2.0))
        budget = float(rng.choice([2e6, 4e6, 8e6])) if rng.random() < budget_fraction else 0.0
        out.append((float(t[i]), k, cam, threshold, budget))
    return out
