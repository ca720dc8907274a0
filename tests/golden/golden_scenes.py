"""Scene and ray-set builders shared by the golden generator and the tests.

Every builder takes a namespace `ns` exposing the scene API (Vec3, Color,
World, Camera, SceneObject, Sphere, Plane, Cube, Mesh, Triangle, IndexedMesh,
Diffuse, Metal, Dielectric, Emissive, Glossy).  make_golden.py passes the
reference's own classes; the tests pass this project's drop-in classes, so
both sides build the scene through identical constructor calls.

Only numpy is imported here so the module loads next to either package.
"""
import numpy as np


def icosphere(subdiv):
    """Unit icosphere: (positions float64 [V,3], faces int32 [F,3])."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.asarray(verts, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.asarray(faces, dtype=np.int64)
    for _ in range(subdiv):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mids])
        nf = len(f)
        a = base + inv[:nf]
        b = base + inv[nf:2 * nf]
        c = base + inv[2 * nf:]
        f = np.concatenate([
            np.stack([f[:, 0], a, c], axis=1),
            np.stack([f[:, 1], b, a], axis=1),
            np.stack([f[:, 2], c, b], axis=1),
            np.stack([a, b, c], axis=1),
        ])
    return v, f.astype(np.int32)


def _tri(ns, a, b, c, group="default"):
    return ns.Triangle(ns.Vec3(*a), ns.Vec3(*b), ns.Vec3(*c), group=group)


def build_trace_scene(ns):
    """Small scene touching every primitive, material and light type."""
    world = ns.World(use_sky=False, background_color=ns.Color(0.05, 0.05, 0.08))
    cam = ns.Camera(position=ns.Vec3(0.5, 0.5, 2.2), forward=ns.Vec3(0, 0, -1),
                    up=ns.Vec3(0, 1, 0), fov=45, width=64, height=64)
    world.add_camera(cam)

    white = ns.Diffuse(ns.Color(0.73, 0.73, 0.73))
    red = ns.Diffuse(ns.Color(0.65, 0.05, 0.05))
    green = ns.Diffuse(ns.Color(0.12, 0.45, 0.15))
    light = ns.Emissive(ns.Color(1.0, 0.9, 0.7), intensity=6.0)

    # box walls as one Mesh of Triangle objects with material groups
    tris = [
        _tri(ns, (0, 1, 0), (1, 1, 0), (1, 1, 1), "white"), _tri(ns, (0, 1, 0), (1, 1, 1), (0, 1, 1), "white"),
        _tri(ns, (0, 0, 0), (1, 0, 0), (1, 1, 0), "white"), _tri(ns, (0, 0, 0), (1, 1, 0), (0, 1, 0), "white"),
        _tri(ns, (0, 0, 0), (0, 1, 0), (0, 1, 1), "red"), _tri(ns, (0, 0, 0), (0, 1, 1), (0, 0, 1), "red"),
        _tri(ns, (1, 0, 0), (1, 0, 1), (1, 1, 1), "green"), _tri(ns, (1, 0, 0), (1, 1, 1), (1, 1, 0), "green"),
        _tri(ns, (0.35, 0.999, 0.35), (0.65, 0.999, 0.35), (0.65, 0.999, 0.65), "light"),
        _tri(ns, (0.35, 0.999, 0.35), (0.65, 0.999, 0.65), (0.35, 0.999, 0.65), "light"),
    ]
    walls = ns.SceneObject(shapes=[ns.Shape(ns.Mesh(tris), {"white": white, "red": red,
                                                            "green": green, "light": light})],
                           name="walls")
    world.add_object(walls)

    # icosphere of Triangle objects with per-vertex normals (glossy), transformed
    pos, faces = icosphere(1)
    ico_tris = []
    for f in faces:
        a, b, c = (ns.Vec3(*[float(x) for x in pos[k]]) for k in f)
        ico_tris.append(ns.Triangle(a, b, c, n0=a, n1=b, n2=c))
    world.add_object(ns.SceneObject(shapes=[ns.Shape(ns.Mesh(ico_tris), {"default": ns.Glossy(ns.Color(0.8, 0.6, 0.3), roughness=0.4)})],
                                    translation=ns.Vec3(0.3, 0.18, 0.35), scale=ns.Vec3(0.15, 0.12, 0.15),
                                    rotation=ns.Vec3(10, 20, 30), name="ico"))

    # analytic primitives
    world.add_object(ns.SceneObject(shape=ns.Sphere(0.12), material=ns.Dielectric(ns.Color(1, 1, 1), ior=1.5),
                                    translation=ns.Vec3(0.7, 0.12, 0.6), name="glass"))
    world.add_object(ns.SceneObject(shape=ns.Sphere(0.1), material=ns.Metal(ns.Color(0.9, 0.9, 0.9), roughness=0.15),
                                    translation=ns.Vec3(0.45, 0.1, 0.7), name="metal"))
    world.add_object(ns.SceneObject(shape=ns.Sphere(1.0), material=ns.Diffuse(ns.Color(0.2, 0.3, 0.8)),
                                    translation=ns.Vec3(0.75, 0.55, 0.3), scale=ns.Vec3(0.08, 0.08, 0.08),
                                    name="blue"))
    world.add_object(ns.SceneObject(shape=ns.Sphere(0.05), material=ns.Emissive(ns.Color(1, 1, 1), intensity=12.0),
                                    translation=ns.Vec3(0.2, 0.8, 0.5), name="bulb"))
    world.add_object(ns.SceneObject(shape=ns.Cube(0.2), material=ns.Diffuse(ns.Color(0.7, 0.7, 0.2)),
                                    translation=ns.Vec3(0.3, 0.1, 0.75), name="cube"))
    world.add_object(ns.SceneObject(shape=ns.Plane(ns.Vec3(0, 1, 0), 0.0), material=white, name="floor"))
    world.add_object(ns.SceneObject(shape=_tri(ns, (0.55, 0.3, 0.2), (0.9, 0.3, 0.25), (0.7, 0.6, 0.2)),
                                    material=ns.Diffuse(ns.Color(0.9, 0.5, 0.5)), name="legacy_tri"))
    return world


def trace_rays(n, seed=7):
    """Camera-like rays from (0.5, 0.5, 2.2) into the box (float32)."""
    rng = np.random.default_rng(seed)
    ro = np.tile(np.array([0.5, 0.5, 2.2], dtype=np.float32), (n, 1))
    tgt = rng.uniform([0.02, 0.02, 0.0], [0.98, 0.98, 0.0], size=(n, 3)).astype(np.float32)
    d = (tgt - ro).astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return ro, d.astype(np.float32)


def soup_triangles(n, seed):
    """Random triangle soup inside [-1, 1]^3 (float32 v0, v1, v2)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, size=(n, 3))
    e = rng.normal(0, 0.08, size=(n, 2, 3))
    v0 = c.astype(np.float32)
    v1 = (c + e[:, 0]).astype(np.float32)
    v2 = (c + e[:, 1]).astype(np.float32)
    return v0, v1, v2


def random_rays(n, seed, spread=1.5):
    rng = np.random.default_rng(seed)
    ro = rng.uniform(-spread, spread, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return ro, d.astype(np.float32)


def build_indexed_object(ns):
    """Transformed IndexedMesh with two material groups and partial normals/uvs."""
    pos, faces = icosphere(2)
    n = len(faces)
    tri_normal_idx = faces.copy()
    tri_normal_idx[::7] = -1          # some triangles fall back to face normals
    uvs = pos[:, :2] * 0.5 + 0.5
    tri_uv_idx = faces.copy()
    tri_uv_idx[::5] = -1
    groups = ["a", "b"]
    tri_group_idx = (np.arange(n) % 3 == 0).astype(np.int32)
    mesh = ns.IndexedMesh(pos * 1.3, faces, normals=pos, tri_normal_idx=tri_normal_idx, uvs=uvs,
                          tri_uv_idx=tri_uv_idx, groups=groups, tri_group_idx=tri_group_idx,
                          build_bvh=False)
    obj = ns.SceneObject(shapes=[ns.Shape(mesh, {"a": ns.Diffuse(ns.Color(0.2, 0.4, 0.6)),
                                                 "b": ns.Metal(ns.Color(0.9, 0.8, 0.7), roughness=0.3)})],
                         translation=ns.Vec3(0.1, -0.2, 0.3), rotation=ns.Vec3(15, -30, 45),
                         scale=ns.Vec3(1.0, 0.5, 2.0), name="indexed")
    return obj


def _surface(ns, tris, indexed):
    """Mesh (Triangle objects) or IndexedMesh of (corners (3,3), uvs (3,2) or
    None, group) triangle specs."""
    if not indexed:
        out = []
        for c, uv, g in tris:
            kw = {} if uv is None else dict(uv0=tuple(uv[0]), uv1=tuple(uv[1]), uv2=tuple(uv[2]))
            out.append(ns.Triangle(*(ns.Vec3(*map(float, p)) for p in c), group=g, **kw))
        return ns.Mesh(out)
    groups = []
    for _, _, g in tris:
        if g not in groups:
            groups.append(g)
    pos = np.concatenate([np.asarray(c, np.float64) for c, _, _ in tris])
    uvs = np.concatenate([np.asarray(uv if uv is not None else np.zeros((3, 2)), np.float64) for _, uv, _ in tris])
    faces = np.arange(3 * len(tris), dtype=np.int32).reshape(-1, 3)
    tri_uv_idx = faces.copy()
    for k, (_, uv, _) in enumerate(tris):
        if uv is None:
            tri_uv_idx[k] = -1
    return ns.IndexedMesh(pos, faces, uvs=uvs, tri_uv_idx=tri_uv_idx, groups=groups,
                          tri_group_idx=[groups.index(g) for _, _, g in tris], build_bvh=False)


def build_texture_scene(ns, indexed=False):
    """Textured surfaces (wrapping, flipped, partial and missing uvs, a
    texture shared by two materials, a textured emitter, an untextured
    triangle with uvs) plus a sphere light, all as Mesh triangles or all as
    IndexedMesh (the reference cannot mix the two in one scene)."""
    rng = np.random.default_rng(60)
    world = ns.World(use_sky=False, background_color=ns.Color(0.05, 0.05, 0.08))
    world.add_camera(ns.Camera(position=ns.Vec3(0.5, 0.5, 2.2), forward=ns.Vec3(0, 0, -1),
                               up=ns.Vec3(0, 1, 0), fov=45, width=64, height=64))
    tex_a = ns.ImageTexture.from_array(rng.random((5, 7, 3)), flip_v=True)
    tex_b = ns.ImageTexture.from_array(rng.integers(0, 256, size=(4, 3, 3)).astype(np.float64), flip_v=False)

    # back wall z = 0: 2x2 quads, uvs wrap past 1, one triangle without uvs
    wall = []
    groups = ["a", "a", "b", "b", "a", "c", "b", "a"]
    k = 0
    for j in range(2):
        for i in range(2):
            x0, y0 = 0.5 * i, 0.5 * j
            quad = [[x0, y0, 0], [x0 + 0.5, y0, 0], [x0 + 0.5, y0 + 0.5, 0], [x0, y0 + 0.5, 0]]
            for tri in ((0, 1, 2), (0, 2, 3)):
                c = np.array([quad[t] for t in tri], np.float64)
                uv = None if k == 5 else c[:, :2] * 2.0 - 0.25
                wall.append((c, uv, groups[k]))
                k += 1
    world.add_object(ns.SceneObject(shapes=[ns.Shape(_surface(ns, wall, indexed), {
        "a": ns.Diffuse(ns.Color(0.9, 0.8, 0.7), albedo_texture=tex_a),
        "b": ns.Glossy(ns.Color(0.7, 0.9, 0.8), roughness=0.4, albedo_texture=tex_b),
        "c": ns.Diffuse(ns.Color(0.6, 0.6, 0.6))})], name="wall"))
    # floor y = 0 (metal sharing texture b, diffuse sharing texture a)
    floor = [(np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1]], np.float64), np.array([[0, 0], [3, 0], [3, 3]]), "f"),
             (np.array([[0, 0, 0], [1, 0, 1], [0, 0, 1]], np.float64), np.array([[0, 0], [3, 3], [0, 3]]), "g")]
    world.add_object(ns.SceneObject(shapes=[ns.Shape(_surface(ns, floor, indexed), {
        "f": ns.Metal(ns.Color(0.8, 0.8, 0.8), roughness=0.2, albedo_texture=tex_b),
        "g": ns.Diffuse(ns.Color(0.5, 0.7, 0.9), albedo_texture=tex_a)})], name="floor"))
    # textured emitter and an untextured triangle that carries uvs
    lamp = [(np.array([[0.2, 0.7, 0.3], [0.45, 0.7, 0.3], [0.2, 0.95, 0.3]]),
             np.array([[0.1, 0.1], [0.9, 0.1], [0.1, 0.9]]), "e"),
            (np.array([[0.6, 0.2, 0.4], [0.9, 0.2, 0.4], [0.6, 0.5, 0.4]]),
             np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), "p")]
    world.add_object(ns.SceneObject(shapes=[ns.Shape(_surface(ns, lamp, indexed), {
        "e": ns.Emissive(ns.Color(1.0, 0.9, 0.8), intensity=4.0, albedo_texture=tex_a),
        "p": ns.Diffuse(ns.Color(0.3, 0.8, 0.3))})], name="lamp"))
    world.add_object(ns.SceneObject(shape=ns.Sphere(0.05), material=ns.Emissive(ns.Color(1, 1, 1), intensity=10.0),
                                    translation=ns.Vec3(0.5, 0.85, 0.6), name="bulb"))
    return world


def texture_rays(n, seed):
    """Camera-like rays from (0.5, 0.5, 2.2) towards the textured wall and floor."""
    rng = np.random.default_rng(seed)
    ro = np.tile(np.array([0.5, 0.5, 2.2], dtype=np.float32), (n, 1))
    tgt = rng.uniform([0.02, -0.3, 0.0], [0.98, 0.98, 0.0], size=(n, 3))
    d = tgt - ro.astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return ro, d.astype(np.float32)
