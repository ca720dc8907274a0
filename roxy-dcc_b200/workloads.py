"""Seeded synthetic scenes for the benchmark configurations.

cornell_box(): unit Cornell box of 36 triangles (5 walls, two rotated boxes,
a 0.25 x 0.25 ceiling light with emission (17, 12, 4)), camera at
(0.5, 0.5, 2.4) looking down -z with a 40 degree FOV.

displaced_icosphere_scene(): icosphere subdivided 7 times (327,680
triangles) with each vertex displaced radially by 3-octave seeded value
noise of amplitude 0.05, 64 analytic spheres of radius U(0.02, 0.1) in a
shell around it, per-object materials (50 % Lambertian U(0.1, 0.9), 30 %
metal fuzz 0.1, 20 % dielectric IOR 1.5), one emissive quad and a uniform
background radiance of 0.2.

All geometry is generated here from a numpy Generator seed; nothing is read
from disk.
"""
import math

import numpy as np

from core import Color, Vec3
from scene import (Camera, Dielectric, Diffuse, Emissive, IndexedMesh, Metal, SceneObject, Shape, Sphere,
                   World)


def icosphere(subdiv):
    """Unit icosphere: (positions float64 [V, 3], faces int32 [F, 3])."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
                  (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * len(v) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a_, b_ = uniq // len(v), uniq % len(v)
        mids = v[a_] + v[b_]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mids])
        nf = len(f)
        m0, m1, m2 = base + inv[:nf], base + inv[nf:2 * nf], base + inv[2 * nf:]
        f = np.concatenate([np.stack([f[:, 0], m0, m2], 1), np.stack([f[:, 1], m1, m0], 1),
                            np.stack([f[:, 2], m2, m1], 1), np.stack([m0, m1, m2], 1)])
    return v, f.astype(np.int32)


def value_noise3(p, seed, octaves=3):
    """Sum of `octaves` lattice value-noise octaves in [-1, 1] (smoothstep
    trilinear interpolation of seeded lattice values)."""
    rng = np.random.default_rng(seed)
    total = np.zeros(len(p))
    norm = 0.0
    for o in range(octaves):
        freq = 2.0 ** (o + 1)
        amp = 0.5 ** o
        lat = rng.uniform(-1.0, 1.0, size=(32, 32, 32))
        q = (p + 2.0) * freq
        i0 = np.floor(q).astype(np.int64)
        fr = q - i0
        s = fr * fr * (3.0 - 2.0 * fr)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) * \
                        (s[:, 2] if dz else 1 - s[:, 2])
                    acc += w * lat[(i0[:, 0] + dx) % 32, (i0[:, 1] + dy) % 32, (i0[:, 2] + dz) % 32]
        total += amp * acc
        norm += amp
    return total / norm


def vertex_normals(pos, faces):
    fn = np.cross(pos[faces[:, 1]] - pos[faces[:, 0]], pos[faces[:, 2]] - pos[faces[:, 0]])
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, faces[:, k], fn)
    vn /= np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-12)
    return vn


def _box_mesh(sx, sy, sz):
    x, y, z = sx / 2, sy / 2, sz / 2
    p = np.array([[-x, -y, -z], [x, -y, -z], [x, y, -z], [-x, y, -z], [-x, -y, z], [x, -y, z], [x, y, z],
                  [-x, y, z]], dtype=np.float64)
    f = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4], [3, 7, 6], [3, 6, 2],
                  [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], dtype=np.int32)
    return p, f


CORNELL = dict(width=256, height=256, samples=16, max_depth=8, fov=40.0)

def cornell_box(width=256, height=256, light_gap=1e-3, light_size=0.25):
    """Config-1 Cornell box (36 triangles); the light hangs `light_gap` below the ceiling."""
    world = World(use_sky=False, background_color=Color(0, 0, 0))
    world.add_camera(Camera(position=Vec3(0.5, 0.5, 2.4), forward=Vec3(0, 0, -1), up=Vec3(0, 1, 0), fov=40,
                            width=width, height=height))
    white = Diffuse(Color(0.73, 0.73, 0.73))
    red = Diffuse(Color(0.65, 0.05, 0.05))
    green = Diffuse(Color(0.12, 0.45, 0.15))
    light = Emissive(Color(17, 12, 4), intensity=1)
    ly = 1.0 - light_gap
    lo, hi = 0.5 - light_size / 2, 0.5 + light_size / 2
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1],          # floor
                    [0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1],          # ceiling
                    [lo, ly, lo], [hi, ly, lo], [hi, ly, hi], [lo, ly, hi]],
                   dtype=np.float64)
    faces = np.array([[0, 2, 1], [0, 3, 2],        # floor
                      [4, 5, 6], [4, 6, 7],        # ceiling
                      [0, 1, 5], [0, 5, 4],        # back (z = 0)
                      [0, 4, 7], [0, 7, 3],        # left (x = 0)
                      [1, 2, 6], [1, 6, 5],        # right (x = 1)
                      [8, 9, 10], [8, 10, 11]],    # light
                     dtype=np.int32)
    groups = ["white", "red", "green", "light"]
    gidx = np.array([0, 0, 0, 0, 0, 0, 1, 1, 2, 2, 3, 3], np.int32)
    walls = IndexedMesh(pos, faces, groups=groups, tri_group_idx=gidx, build_bvh=False)
    world.add_object(SceneObject(shapes=[Shape(walls, {"white": white, "red": red, "green": green,
                                                       "light": light})], name="walls"))
    tp, tf = _box_mesh(0.3, 0.6, 0.3)
    world.add_object(SceneObject(shapes=[Shape(IndexedMesh(tp, tf, build_bvh=False), {"default": white})],
                                 translation=Vec3(0.32, 0.3, 0.34), rotation=Vec3(0, 15, 0), name="tall"))
    sp, sf = _box_mesh(0.3, 0.3, 0.3)
    world.add_object(SceneObject(shapes=[Shape(IndexedMesh(sp, sf, build_bvh=False), {"default": white})],
                                 translation=Vec3(0.68, 0.15, 0.64), rotation=Vec3(0, -18, 0), name="short"))
    return world


ICOSPHERE_SCENE = dict(width=1920, height=1080, samples=64, max_depth=12, fov=45.0)


def _draw_material(rng):
    u = rng.random()
    if u < 0.5:
        return Diffuse(Color(*[float(x) for x in rng.uniform(0.1, 0.9, 3)]))
    if u < 0.8:
        return Metal(Color(0.9, 0.9, 0.9), roughness=0.1)
    return Dielectric(Color(1.0, 1.0, 1.0), ior=1.5)


def displaced_icosphere_scene(width=1920, height=1080, subdiv=7, n_spheres=64, seed=2024):
    """Config-2 scene: 327,680-triangle displaced icosphere + 64 spheres."""
    rng = np.random.default_rng(seed)
    pos, faces = icosphere(subdiv)
    disp = 0.05 * value_noise3(pos, seed + 1)
    pos = pos * (1.0 + disp)[:, None]
    nrm = vertex_normals(pos, faces)
    world = World(use_sky=False, background_color=Color(0.2, 0.2, 0.2))
    world.add_camera(Camera(position=Vec3(0.0, 0.35, 3.4), forward=Vec3(0, -0.1, -1), up=Vec3(0, 1, 0), fov=45,
                            width=width, height=height))
    mesh = IndexedMesh(pos, faces, normals=nrm, tri_normal_idx=faces, build_bvh=False)
    world.add_object(SceneObject(shapes=[Shape(mesh, {"default": _draw_material(rng)})], name="icosphere"))
    for i in range(n_spheres):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        r = float(rng.uniform(0.02, 0.1))
        c = d * rng.uniform(1.15, 1.6)
        world.add_object(SceneObject(shape=Sphere(r), material=_draw_material(rng),
                                     translation=Vec3(*[float(x) for x in c]), name=f"sphere{i}"))
    q = 0.75
    lp = np.array([[-q, 2.4, -q], [q, 2.4, -q], [q, 2.4, q], [-q, 2.4, q]], dtype=np.float64)
    lf = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)
    world.add_object(SceneObject(shapes=[Shape(IndexedMesh(lp, lf, build_bvh=False),
                                               {"default": Emissive(Color(1.0, 0.95, 0.85), intensity=15.0)})],
                                 name="light"))
    return world


BOX_COLORS = [(0.73, 0.73, 0.73), (0.65, 0.05, 0.05), (0.12, 0.45, 0.15)]


def instanced_box_scene(n_tris, seed, width=256, height=256, n_spheres=16):
    """One scene of the batched configuration: seeded instances of a unit box
    (12 triangles each, n_tris // 12 of them, random size, yaw and
    position) in one IndexedMesh with the Cornell box's three Lambertian
    albedos as material groups, `n_spheres` Lambertian spheres, a floor quad
    and a 0.5 x 0.5 emissive quad with emission (17, 12, 4)."""
    rng = np.random.default_rng(seed)
    n_box = max(1, n_tris // 12)
    bp, bf = _box_mesh(1.0, 1.0, 1.0)
    size = rng.uniform(0.02, 0.12, size=(n_box, 3)) * (1.0 + 3.0 * (n_box < 400))
    yaw = rng.uniform(0.0, 2.0 * np.pi, n_box)
    spread = 1.0 + 0.25 * np.log10(n_box)
    ctr = np.stack([rng.uniform(-spread, spread, n_box), rng.uniform(0.0, 1.2, n_box),
                    rng.uniform(-spread, spread, n_box)], axis=1)
    c, s = np.cos(yaw), np.sin(yaw)
    local = bp[None, :, :] * size[:, None, :]
    x = c[:, None] * local[:, :, 0] + s[:, None] * local[:, :, 2]
    z = -s[:, None] * local[:, :, 0] + c[:, None] * local[:, :, 2]
    pos = np.stack([x, local[:, :, 1], z], axis=2) + ctr[:, None, :]
    faces = (bf[None, :, :] + 8 * np.arange(n_box, dtype=np.int32)[:, None, None]).reshape(-1, 3)
    gidx = np.repeat(rng.integers(0, 3, n_box).astype(np.int32), 12)
    world = World(use_sky=False, background_color=Color(0.0, 0.0, 0.0))
    world.add_camera(Camera(position=Vec3(0.0, 1.6, 2.6 * spread + 1.0), forward=Vec3(0, -0.45, -1),
                            up=Vec3(0, 1, 0), fov=40, width=width, height=height))
    mats = {f"c{k}": Diffuse(Color(*BOX_COLORS[k])) for k in range(3)}
    mesh = IndexedMesh(pos.reshape(-1, 3), faces, groups=list(mats), tri_group_idx=gidx, build_bvh=False)
    world.add_object(SceneObject(shapes=[Shape(mesh, mats)], name="boxes"))
    for i in range(n_spheres):
        r = float(rng.uniform(0.05, 0.2))
        p = [float(rng.uniform(-spread, spread)), r, float(rng.uniform(-spread, spread))]
        world.add_object(SceneObject(shape=Sphere(r), material=Diffuse(Color(*BOX_COLORS[i % 3])),
                                     translation=Vec3(*p), name=f"sphere{i}"))
    e = 2.0 * spread
    fp = np.array([[-e, 0, -e], [e, 0, -e], [e, 0, e], [-e, 0, e]], dtype=np.float64)
    world.add_object(SceneObject(shapes=[Shape(IndexedMesh(fp, np.array([[0, 2, 1], [0, 3, 2]], np.int32),
                                                           build_bvh=False), {"default": Diffuse(Color(*BOX_COLORS[0]))})],
                                 name="floor"))
    lp = np.array([[-0.25, 2.5, -0.25], [0.25, 2.5, -0.25], [0.25, 2.5, 0.25], [-0.25, 2.5, 0.25]], np.float64)
    world.add_object(SceneObject(shapes=[Shape(IndexedMesh(lp, np.array([[0, 1, 2], [0, 2, 3]], np.int32),
                                                           build_bvh=False),
                                               {"default": Emissive(Color(17.0, 12.0, 4.0), intensity=1.0)})],
                                 name="light"))
    return world


def batch_specs(n_scenes=64, seed=7, tri_range=(1e3, 2e6), resolutions=(256, 512, 1024), spps=(1, 4, 16, 64),
                depth_range=(4, 16)):
    """The batched configuration: per scene a triangle count log-uniform in
    `tri_range`, a square resolution, spp and max depth drawn by seed."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_scenes):
        n = int(round(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))))
        res = int(rng.choice(resolutions))
        specs.append(dict(n_tris=n, width=res, height=res, spp=int(rng.choice(spps)),
                          max_depth=int(rng.integers(depth_range[0], depth_range[1] + 1)), seed=seed * 1000 + i))
    return specs


def camera_params(world, width, height):
    cam = world.active_camera
    return dict(fov_tan=math.tan(math.radians(cam.fov) / 2), aspect=cam.aspect_ratio, cam_pos=list(cam.position),
                cam_fwd=list(cam.forward), cam_right=list(cam.right), cam_up=list(cam.up))


def obj_text(copies=8, subdiv=7, seed=2024):
    """The OBJ-ingestion workload: `copies` translated instances of the
    displaced icosphere (327,680 triangles each at subdiv 7) as Wavefront
    text, written the way exporters write it: one `o` and `usemtl` per copy,
    `v` / `vn` rows with six decimals, faces as v//vn triples.  Seeded; with
    8 copies about 2.6 M triangles in 190 MB of text."""
    pos, faces = icosphere(subdiv)
    pos = pos * (1.0 + 0.05 * value_noise3(pos, seed + 1))[:, None]
    nrm = vertex_normals(pos, faces)
    nv = len(pos)
    vn_lines = "\n".join(f"vn {a:.6f} {b:.6f} {c:.6f}" for a, b, c in nrm.tolist())
    out = ["# displaced icosphere x %d, seed %d" % (copies, seed)]
    for k in range(copies):
        p = pos + np.array([2.5 * (k % 4), 0.0, 2.5 * (k // 4)])
        out.append(f"o sphere{k}")
        out.append("\n".join(f"v {a:.6f} {b:.6f} {c:.6f}" for a, b, c in p.tolist()))
        out.append(vn_lines)
        out.append(f"usemtl mat{k % 3}")
        f = faces + 1 + k * nv
        out.append("\n".join(f"f {a}//{a} {b}//{b} {c}//{c}" for a, b, c in f.tolist()))
    return ("\n".join(out) + "\n").encode("ascii")
