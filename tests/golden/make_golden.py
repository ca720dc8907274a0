"""Generate the golden vectors under tests/golden/ from the reference itself.

Run in a container that has the reference checkout:

    python tests/golden/make_golden.py /path/to/roxy-dcc

The reference's Python is imported with the import-only stand-ins in
`_refshim/` (taichi, pygame, moderngl).  Its `@ti.func` bodies then run as
plain float32 Python, so every golden number below is produced by the
reference's own source:

  bvh_build.npz   GPUBVHBuilder.build              (rendering/taichi/bvh_builder.py:315-544)
  traversal.npz   bvh_intersect / bvh_occluded     (rendering/taichi/intersect.py:81-219)
  prims.npz       Sphere/Plane/Cube/Triangle.taichi_intersect (scene/primitives.py:90-215,
                  scene/mesh.py:133-157)
  trace_scene.npz extract_scene output, scene_intersect and trace() with a scripted
                  random stream                    (rendering/taichi/extractor.py,
                                                    intersect.py:249-309, trace.py:139-236)
  denoise.npz     edge_aware_denoise               (rendering/denoise.py:23-104)
  sampling.npz    pixel_sample_offset              (rendering/sampling.py:17-23)

Nothing at test time reads the reference; the tests read these fixtures.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _setup(ref_root):
    sys.path.insert(0, os.path.join(HERE, "_refshim"))
    sys.path.insert(1, ref_root)
    sys.path.insert(2, HERE)
    sys.setrecursionlimit(100000)


def _ns():
    import core
    import scene
    from scene.materials import Emissive, Glossy

    class NS:
        pass

    ns = NS()
    for name in ("Vec3", "Color"):
        setattr(ns, name, getattr(core, name))
    for name in ("World", "Camera", "SceneObject", "Sphere", "Plane", "Cube", "Mesh", "Triangle",
                 "IndexedMesh", "Diffuse", "Metal", "Dielectric", "Shape"):
        setattr(ns, name, getattr(scene, name))
    ns.Emissive = Emissive
    ns.Glossy = Glossy
    ns.ImageTexture = scene.ImageTexture
    return ns


def _tri_dict(x):
    return {'v0': [x, 0, 0], 'v1': [x + 1, 0, 0], 'v2': [x, 1, 0],
            'n0': [0, 0, 1], 'n1': [0, 0, 1], 'n2': [0, 0, 1],
            'mat_type': 0, 'albedo': [1, 1, 1], 'roughness': 0.0, 'ior': 1.0, 'emission': 0.0}


def _nodes_arrays(builder):
    nodes = builder.nodes
    n = len(nodes)
    out = {
        "node_min": np.array([nd['aabb_min'] for nd in nodes], dtype=np.float32).reshape(n, 3),
        "node_max": np.array([nd['aabb_max'] for nd in nodes], dtype=np.float32).reshape(n, 3),
        "left": np.array([nd['left'] for nd in nodes], dtype=np.int32),
        "right": np.array([nd['right'] for nd in nodes], dtype=np.int32),
        "start": np.array([nd['tri_start'] for nd in nodes], dtype=np.int32),
        "count": np.array([nd['tri_count'] for nd in nodes], dtype=np.int32),
        "order": np.asarray(builder.ordered_tris, dtype=np.int32),
    }
    return out


def make_bvh(out_dir):
    from rendering.taichi.bvh_builder import GPUBVHBuilder, TriangleBatch
    import golden_scenes as gs

    cases = {}

    def add(name, v0, v1, v2, leaf):
        n = len(v0)
        batch = TriangleBatch(v0, v1, v2,
                              np.tile([0, 0, 1], (n, 1)), np.tile([0, 0, 1], (n, 1)), np.tile([0, 0, 1], (n, 1)),
                              np.zeros(n, np.int32), np.ones((n, 3), np.float32), np.zeros(n, np.float32),
                              np.ones(n, np.float32), np.zeros(n, np.float32))
        b = GPUBVHBuilder()
        b.MAX_LEAF_SIZE = leaf
        b.build([batch])
        arr = _nodes_arrays(b)
        cases[name] = dict(v0=np.asarray(v0, np.float32), v1=np.asarray(v1, np.float32),
                           v2=np.asarray(v2, np.float32), leaf=np.int32(leaf), **arr)

    for name, xs, leaf in (("legacy_perm_leaf1", [7, 1, 6, 0, 5, 2, 4, 3], 1),
                           ("legacy_range_leaf4", list(range(8)), 4),
                           ("legacy_two_leaf8", [0, 2], 8)):
        d = [_tri_dict(x) for x in xs]
        add(name, [t['v0'] for t in d], [t['v1'] for t in d], [t['v2'] for t in d], leaf)
    for n, leaf, seed in ((1, 8, 1), (2, 8, 2), (9, 8, 3), (100, 8, 4), (1000, 8, 5), (5000, 8, 6),
                          (3000, 4, 7), (777, 1, 8), (4096, 2, 9)):
        v0, v1, v2 = gs.soup_triangles(n, seed)
        add(f"soup{n}_leaf{leaf}", v0, v1, v2, leaf)
    pos, f = gs.icosphere(3)
    add("ico3_leaf8", pos[f[:, 0]].astype(np.float32), pos[f[:, 1]].astype(np.float32),
        pos[f[:, 2]].astype(np.float32), 8)
    # flat in z: zero centroid extent on one axis
    v0, v1, v2 = gs.soup_triangles(300, 10)
    for v in (v0, v1, v2):
        v[:, 2] = 0.25
    add("flat300_leaf8", v0, v1, v2, 8)
    # duplicated triangles: equal Morton codes, order decided by the stable sort
    v0, v1, v2 = gs.soup_triangles(40, 11)
    add("dup200_leaf3", np.repeat(v0, 5, 0), np.repeat(v1, 5, 0), np.repeat(v2, 5, 0), 3)

    flat = {}
    for name, d in cases.items():
        for k, v in d.items():
            flat[f"{name}/{k}"] = v
    flat["case_names"] = np.array(sorted(cases))
    np.savez_compressed(os.path.join(out_dir, "bvh_build.npz"), **flat)

    # palette / material dedupe behaviour (bvh_builder.py:370-410)
    batch = TriangleBatch.from_dicts([_tri_dict(0), dict(_tri_dict(2), albedo=[0.5, 0.5, 0.5]),
                                      dict(_tri_dict(4), mat_type=1, roughness=0.25), _tri_dict(6)])
    b = GPUBVHBuilder().build([batch])
    np.savez_compressed(os.path.join(out_dir, "bvh_palette.npz"),
                        ordered_mat_idx=b._ordered_mat_idx.astype(np.int32),
                        palette_type=np.array([m['type'] for m in b.mat_palette], np.int32),
                        palette_albedo=np.array([m['albedo'] for m in b.mat_palette], np.float32),
                        palette_roughness=np.array([m['roughness'] for m in b.mat_palette], np.float32))
    print("bvh_build.npz:", len(cases), "cases")


def _load_reference_bvh(batch, leaf):
    from rendering.taichi.bvh_builder import GPUBVHBuilder
    b = GPUBVHBuilder()
    b.MAX_LEAF_SIZE = leaf
    b.build([batch])
    b.upload()
    return b


def make_traversal(out_dir):
    import taichi as ti
    from rendering.taichi.bvh_builder import TriangleBatch
    import rendering.taichi.intersect as isect
    import rendering.taichi.fields as fields
    import golden_scenes as gs

    out = {}
    for case, (v0, v1, v2), leaf, (ro, rd) in (
        ("soup2000", gs.soup_triangles(2000, 21), 8, gs.random_rays(400, 22)),
        ("ico3", tuple(np.asarray(x, np.float32) for x in _ico_tris(3)), 4, gs.random_rays(300, 23, spread=2.0)),
    ):
        n = len(v0)
        batch = TriangleBatch(v0, v1, v2, np.tile([0, 0, 1], (n, 1)), np.tile([0, 0, 1], (n, 1)),
                              np.tile([0, 0, 1], (n, 1)), np.zeros(n, np.int32), np.ones((n, 3)),
                              np.zeros(n), np.ones(n), np.zeros(n))
        b = _load_reference_bvh(batch, leaf)
        fields._bvh_n_tris[None] = b.triangle_count
        ts, ids, us, vs, occ = [], [], [], [], []
        rng = np.random.default_rng(99)
        max_t = rng.uniform(0.05, 3.0, size=len(ro)).astype(np.float32)
        for i in range(len(ro)):
            t, idx, u, v = isect.bvh_intersect(ti.Vector(ro[i]), ti.Vector(rd[i]))
            ts.append(np.float32(t)); ids.append(int(idx)); us.append(np.float32(u)); vs.append(np.float32(v))
            occ.append(int(isect.bvh_occluded(ti.Vector(ro[i]), ti.Vector(rd[i]), max_t[i])))
        arr = _nodes_arrays(b)
        out.update({f"{case}/v0": v0, f"{case}/v1": v1, f"{case}/v2": v2, f"{case}/leaf": np.int32(leaf),
                    f"{case}/ro": ro, f"{case}/rd": rd, f"{case}/max_t": max_t,
                    f"{case}/t": np.array(ts, np.float32), f"{case}/idx": np.array(ids, np.int32),
                    f"{case}/u": np.array(us, np.float32), f"{case}/v": np.array(vs, np.float32),
                    f"{case}/occluded": np.array(occ, np.int32)})
        out.update({f"{case}/{k}": v for k, v in arr.items()})
        print(f"traversal {case}: {len(ro)} rays, hits={int(np.sum(np.array(ids) >= 0))}")
    out["case_names"] = np.array(["soup2000", "ico3"])
    np.savez_compressed(os.path.join(out_dir, "traversal.npz"), **out)


def _ico_tris(subdiv):
    import golden_scenes as gs
    pos, f = gs.icosphere(subdiv)
    pos = pos * 0.9
    return pos[f[:, 0]], pos[f[:, 1]], pos[f[:, 2]]


def make_prims(out_dir):
    import taichi as ti
    from scene.primitives import Sphere, Plane, Cube
    from scene.mesh import Triangle
    import golden_scenes as gs

    ro, rd = gs.random_rays(300, 31, spread=1.2)
    rng = np.random.default_rng(32)
    cen = rng.uniform(-0.5, 0.5, size=(300, 3)).astype(np.float32)
    rad = rng.uniform(0.1, 0.9, size=300).astype(np.float32)
    nrm = rng.normal(size=(300, 3))
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    off = rng.uniform(-1, 1, size=300).astype(np.float32)
    he = rng.uniform(0.1, 0.6, size=(300, 3)).astype(np.float32)
    v0, v1, v2 = gs.soup_triangles(300, 33)
    v1 = (v0 + (v1 - v0) * 8).astype(np.float32)
    v2 = (v0 + (v2 - v0) * 8).astype(np.float32)
    ts = {"sphere": [], "plane": [], "cube": [], "tri": [], "cube_normal": []}
    for i in range(300):
        o, d = ti.Vector(ro[i]), ti.Vector(rd[i])
        ts["sphere"].append(np.float32(Sphere.taichi_intersect(o, d, ti.Vector(cen[i]), rad[i])))
        ts["plane"].append(np.float32(Plane.taichi_intersect(o, d, ti.Vector(nrm[i]), off[i])))
        with np.errstate(divide="ignore", invalid="ignore"):
            tc = Cube.taichi_intersect(o, d, ti.Vector(cen[i]), ti.Vector(he[i]))
        ts["cube"].append(np.float32(tc))
        hp = o + d * np.float32(tc if tc > 0 else 1.0)
        ts["cube_normal"].append(Cube.taichi_normal(hp, ti.Vector(cen[i]), ti.Vector(he[i])).to_list())
        ts["tri"].append(np.float32(Triangle.taichi_intersect(o, d, ti.Vector(v0[i]), ti.Vector(v1[i]), ti.Vector(v2[i]))))
    np.savez_compressed(os.path.join(out_dir, "prims.npz"), ro=ro, rd=rd, center=cen, radius=rad, normal=nrm,
                        offset=off, half=he, v0=v0, v1=v1, v2=v2,
                        **{f"t_{k}": np.array(v, np.float32) for k, v in ts.items()})
    print("prims.npz written")


def _dump_field(fld, n, width=None, dtype=np.float32):
    out = np.zeros((n, width) if width else (n,), dtype=dtype)
    for i in range(n):
        v = fld[i]
        out[i] = v.e if hasattr(v, "e") else v
    return out


def make_trace_scene(out_dir):
    import taichi as ti
    import rendering.taichi.fields as F
    import rendering.taichi.trace  # noqa: F401 (the package re-exports a function of the same name)
    trace_mod = sys.modules["rendering.taichi.trace"]
    import rendering.taichi.intersect as isect
    from rendering.taichi.extractor import extract_scene
    import golden_scenes as gs

    world = gs.build_trace_scene(_ns())
    stats = extract_scene(world)
    out = _dump_scene(F, stats)
    # scene_intersect on camera-like rays
    ro, rd = gs.trace_rays(300, seed=41)
    si = {"t": [], "idx": [], "is_bvh": [], "u": [], "v": [], "normal": []}
    for i in range(len(ro)):
        t, nrm, idx, is_bvh, _mat, u, v = isect.scene_intersect(ti.Vector(ro[i]), ti.Vector(rd[i]))
        si["t"].append(np.float32(t)); si["idx"].append(int(idx)); si["is_bvh"].append(int(is_bvh))
        si["u"].append(np.float32(u)); si["v"].append(np.float32(v)); si["normal"].append(nrm.to_list())
    out.update({"si_ro": ro, "si_rd": rd})
    out.update({f"si_{k}": np.array(v, np.float32 if k in ("t", "u", "v", "normal") else np.int32)
                for k, v in si.items()})
    out.update(_scripted_traces(trace_mod, gs.trace_rays(96, seed=42), seed=43,
                                configs=[(6, 0, 0, 1), (6, 0, 1, 3), (8, 1, 0, 8), (1, 0, 0, 0)]))
    np.savez_compressed(os.path.join(out_dir, "trace_scene.npz"), **out)

    # IndexedMesh flattening (scene/mesh.py:397-430 via extractor.py:174-191)
    obj = gs.build_indexed_object(_ns())
    geo = obj.shapes[0].geometry
    arrs = geo.indexed_triangle_arrays(obj.world_matrix, obj.world_inverse_transpose_matrix)
    np.savez_compressed(os.path.join(out_dir, "indexed_arrays.npz"),
                        **{k: np.asarray(v) for k, v in arrs.items() if k != "groups"},
                        world_matrix=np.array(obj.world_matrix.rows, np.float64),
                        world_inverse=np.array(obj.world_inverse_matrix.rows, np.float64))
    print(f"trace_scene.npz: stats={list(out['stats'])}")


def _scripted_traces(trace_mod, rays, seed, configs):
    """trace() with scripted ti.random() streams, per (max_depth, use_sky,
    direct_light_mode, direct_light_max_depth) config and ray."""
    import taichi as ti
    counter = ti.CounterField()
    trace_mod._ray_count = counter
    tro, trd = rays
    rng = np.random.default_rng(seed)
    recs = {k: [] for k in ("color", "normal", "albedo", "depth", "consumed", "rays", "cfg")}
    streams = []
    bg = ti.Vector([0.05, 0.05, 0.08])
    for ci, (md, sky, mode, dlmd) in enumerate(configs):
        for i in range(len(tro)):
            stream = rng.random(512).astype(np.float32)
            ti.set_random_stream(stream)
            counter.value = 0
            color, nrm, alb, dep = trace_mod.trace(ti.Vector(tro[i]), ti.Vector(trd[i]), md, sky, bg,
                                                   mode, dlmd, 1)
            recs["color"].append(color.to_list()); recs["normal"].append(nrm.to_list())
            recs["albedo"].append(alb.to_list()); recs["depth"].append(float(dep))
            recs["consumed"].append(ti.consumed()); recs["rays"].append(counter.value)
            recs["cfg"].append(ci)
            streams.append(stream)
    out = {"tr_ro": np.tile(tro, (len(configs), 1)), "tr_rd": np.tile(trd, (len(configs), 1)),
           "tr_stream": np.array(streams, np.float32), "tr_configs": np.array(configs, np.int32),
           "tr_bg": np.array([0.05, 0.05, 0.08], np.float32)}
    for k, v in recs.items():
        out[f"tr_{k}"] = np.array(v, np.float32 if k in ("color", "normal", "albedo", "depth") else np.int32)
    return out


def make_texture_scene(out_dir):
    for indexed, name in ((False, "texture_scene.npz"), (True, "texture_scene_indexed.npz")):
        _make_texture_scene(out_dir, indexed, name)


def _make_texture_scene(out_dir, indexed, name):
    """Textured scene: extract_scene's uv / texture fields, _sample_texture,
    _bvh_albedo and trace() with scripted random streams."""
    import taichi as ti
    import rendering.taichi.fields as F
    import rendering.taichi.trace  # noqa: F401
    trace_mod = sys.modules["rendering.taichi.trace"]
    from rendering.taichi.extractor import extract_scene
    import golden_scenes as gs

    world = gs.build_texture_scene(_ns(), indexed=indexed)
    stats = extract_scene(world)
    out = _dump_scene(F, stats)
    n_tris = int(F._bvh_n_tris[None])
    n_mats = int(F._mat_n_mats[None])
    n_tex = int(F._tex_n[None])
    out.update({"uv0": _dump_field(F._bvh_uv0, n_tris, 2), "uv1": _dump_field(F._bvh_uv1, n_tris, 2),
                "uv2": _dump_field(F._bvh_uv2, n_tris, 2),
                "has_uv": _dump_field(F._bvh_has_uv, n_tris, dtype=np.int32),
                "mat_texture": _dump_field(F._mat_texture, n_mats, dtype=np.int32),
                "tex_w": _dump_field(F._tex_width, n_tex, dtype=np.int32),
                "tex_h": _dump_field(F._tex_height, n_tex, dtype=np.int32),
                "tex_flip": _dump_field(F._tex_flip_v, n_tex, dtype=np.int32)})
    for i in range(n_tex):
        out[f"tex{i}"] = np.array(F._tex_pixels.data[i, :out["tex_h"][i], :out["tex_w"][i]], np.uint8)
    # _sample_texture over wrapped, negative and edge uvs
    rng = np.random.default_rng(61)
    uv = rng.uniform(-2.5, 2.5, size=(300, 2)).astype(np.float32)
    uv[:8] = [[0, 0], [1, 1], [0.999999, 0.5], [-1e-7, 0.25], [0.5, -0.0], [2.0, -3.0], [0.25, 0.75],
              [-0.5, 1.5]]
    samp = []
    for t in range(n_tex):
        samp.append([trace_mod._sample_texture(t, ti.Vector(list(x))).to_list() for x in uv])
    out["st_uv"] = uv
    out["st_out"] = np.array(samp, np.float32)
    # _bvh_albedo on every BVH triangle at seeded barycentrics
    bu = rng.uniform(0, 0.5, n_tris).astype(np.float32)
    bv = rng.uniform(0, 0.5, n_tris).astype(np.float32)
    ba = []
    for i in range(n_tris):
        m = int(F._bvh_mat_idx[i])
        ba.append(trace_mod._bvh_albedo(i, m, bu[i], bv[i], F._mat_albedo[m]).to_list())
    out.update({"ba_u": bu, "ba_v": bv, "ba_out": np.array(ba, np.float32)})
    out.update(_scripted_traces(trace_mod, gs.texture_rays(80, seed=62), seed=63,
                                configs=[(6, 0, 0, 1), (5, 1, 1, 3)]))
    np.savez_compressed(os.path.join(out_dir, name), **out)
    print(f"{name}: stats={list(out['stats'])} textures={n_tex}")


def _dump_scene(F, stats):
    n_obj = int(F._n_objects[None])
    n_nodes = int(F._bvh_n_nodes[None])
    n_tris = int(F._bvh_n_tris[None])
    n_mats = int(F._mat_n_mats[None])
    n_lights = int(F._n_lights[None])
    out = {
        "stats": np.array([stats['primitive_count'], stats['bvh_nodes'], stats['bvh_triangles'],
                           stats['bvh_materials'], stats['bvh_leaf_size']], np.int32),
        "obj_type": _dump_field(F._obj_type, n_obj, dtype=np.int32),
        "obj_center": _dump_field(F._obj_center, n_obj, 3),
        "obj_radius": _dump_field(F._obj_radius, n_obj),
        "obj_normal": _dump_field(F._obj_normal, n_obj, 3),
        "obj_offset": _dump_field(F._obj_offset, n_obj),
        "obj_extra": _dump_field(F._obj_extra, n_obj, 3),
        "obj_v0": _dump_field(F._obj_v0, n_obj, 3),
        "obj_v1": _dump_field(F._obj_v1, n_obj, 3),
        "obj_v2": _dump_field(F._obj_v2, n_obj, 3),
        "obj_mat_type": _dump_field(F._obj_mat_type, n_obj, dtype=np.int32),
        "obj_albedo": _dump_field(F._obj_albedo, n_obj, 3),
        "obj_roughness": _dump_field(F._obj_roughness, n_obj),
        "obj_ior": _dump_field(F._obj_ior, n_obj),
        "obj_emission": _dump_field(F._obj_emission, n_obj),
        "light_center": _dump_field(F._light_center, n_lights, 3),
        "light_radius": _dump_field(F._light_radius, n_lights),
        "light_albedo": _dump_field(F._light_albedo, n_lights, 3),
        "light_emission": _dump_field(F._light_emission, n_lights),
        "node_min": _dump_field(F._bvh_aabb_min, n_nodes, 3),
        "node_max": _dump_field(F._bvh_aabb_max, n_nodes, 3),
        "left": _dump_field(F._bvh_left, n_nodes, dtype=np.int32),
        "right": _dump_field(F._bvh_right, n_nodes, dtype=np.int32),
        "start": _dump_field(F._bvh_tri_start, n_nodes, dtype=np.int32),
        "count": _dump_field(F._bvh_tri_count, n_nodes, dtype=np.int32),
        "v0": _dump_field(F._bvh_v0, n_tris, 3), "v1": _dump_field(F._bvh_v1, n_tris, 3),
        "v2": _dump_field(F._bvh_v2, n_tris, 3),
        "n0": _dump_field(F._bvh_n0, n_tris, 3), "n1": _dump_field(F._bvh_n1, n_tris, 3),
        "n2": _dump_field(F._bvh_n2, n_tris, 3),
        "tri_mat": _dump_field(F._bvh_mat_idx, n_tris, dtype=np.int32),
        "mat_type": _dump_field(F._mat_type, n_mats, dtype=np.int32),
        "mat_albedo": _dump_field(F._mat_albedo, n_mats, 3),
        "mat_roughness": _dump_field(F._mat_roughness, n_mats),
        "mat_ior": _dump_field(F._mat_ior, n_mats),
        "mat_emission": _dump_field(F._mat_emission, n_mats),
    }
    return out


def make_denoise(out_dir):
    from rendering.denoise import edge_aware_denoise, linear_to_display
    rng = np.random.default_rng(51)
    out = {}
    cases = [
        ("small_color_only", (5, 5), 1, 0.2, 0.8, None),
        ("legacy_none", (4, 5), 1, 0.25, 0.6, None),
        ("r1_all_guides", (37, 53), 1, 0.08, 0.8, ("normal", "albedo", "depth")),
        ("r2_all_guides", (40, 31), 2, 0.3, 1.0, ("normal", "albedo", "depth")),
        ("r1_normal_only", (33, 33), 1, 0.5, 0.7, ("normal",)),
        ("r3_albedo_depth", (29, 45), 3, 0.15, 0.9, ("albedo", "depth")),
        ("r1_hdr", (64, 48), 1, 0.08, 0.8, ("normal", "albedo", "depth")),
    ]
    names = []
    for name, (h, w), r, sc, amt, guides in cases:
        px = rng.random((h, w, 3), dtype=np.float32)
        if name == "r1_hdr":
            px = (px * 12.0).astype(np.float32)
        kw = {}
        if guides:
            if "normal" in guides:
                nrm = rng.normal(size=(h, w, 3)).astype(np.float32)
                nrm /= np.linalg.norm(nrm, axis=2, keepdims=True)
                nrm[: h // 2] = [0, 1, 0]
                kw["normal"] = nrm.astype(np.float32)
            if "albedo" in guides:
                alb = rng.random((h, w, 3), dtype=np.float32)
                alb[:, : w // 3] = 0.5
                kw["albedo"] = alb
            if "depth" in guides:
                kw["depth"] = (rng.random((h, w), dtype=np.float32) * 4.0 + 1.0).astype(np.float32)
        res = edge_aware_denoise(px, radius=r, sigma_color=sc, amount=amt, **kw)
        out[f"{name}/pixels"] = px
        for k, v in kw.items():
            out[f"{name}/{k}"] = v
        out[f"{name}/params"] = np.array([r, sc, amt], np.float64)
        out[f"{name}/out"] = np.asarray(res, np.float32)
        names.append(name)
    lin = rng.normal(0.5, 0.6, size=(16, 16, 3)).astype(np.float32)
    out["display/in"] = lin
    out["display/out"] = linear_to_display(lin)
    out["case_names"] = np.array(names)
    np.savez_compressed(os.path.join(out_dir, "denoise.npz"), **out)
    print("denoise.npz:", len(names), "cases")


def make_sampling(out_dir):
    from rendering.sampling import pixel_sample_offset
    vals = np.zeros((16, 16, 8, 2), np.float64)
    for y in range(16):
        for x in range(16):
            for f in range(8):
                vals[y, x, f] = pixel_sample_offset(x, y, f)
    np.savez_compressed(os.path.join(out_dir, "sampling.npz"), offsets=vals)
    print("sampling.npz written")


def _obj_num(rng, x):
    """One number in one of the spellings OBJ exporters and people write."""
    k = int(rng.integers(0, 10))
    if k == 0:
        return f"{x:.6f}"
    if k == 1:
        return f"{x:.3e}"
    if k == 2:
        return repr(float(x))  # up to 17 significant digits
    if k == 3:
        return f"{x:+.4f}"
    if k == 4:
        return f"{x:.9g}"
    if k == 5:
        return f"{x:.2E}"
    if k == 6:
        return str(int(round(x)))
    if k == 7:
        return f"{x:.1f}".replace("0.", ".", 1) if abs(x) < 1 and x >= 0 else f"{x:.1f}"
    if k == 8:
        return f"{x:.22f}"  # too many digits for the device's exact path
    return f"{x:.5f}"


def _obj_text(seed, n_blocks):
    """Seeded OBJ text covering the reader's cases: v with extra components,
    vt with 2 and 3, vn; faces of 2..6 vertices in every index form
    (v, v/t, v//n, v/t/n, v/t/n/extra), absolute and relative indices;
    usemtl runs (repeated, unnamed, non-ASCII); o / g / s / mtllib;
    comments, blank lines, tabs, CRLF and lone CR endings; unrecognised
    keywords; numbers with exponents, signs, long digit strings, inf / nan
    and underscores."""
    rng = np.random.default_rng(seed)
    out = ["# synthetic OBJ, seed %d" % seed, "mtllib not_there.mtl", "", "o Body", "g part0", "s off"]
    nv = nvt = nvn = 0
    mats = ["red", "green", "blue", "steel", "mat_été", "red"]
    for b in range(n_blocks):
        for _ in range(int(rng.integers(3, 9))):
            xs = rng.normal(size=4) * 10.0 ** rng.integers(-3, 3)
            extra = " " + _obj_num(rng, xs[3]) if rng.random() < 0.1 else ""
            out.append("v " + " ".join(_obj_num(rng, x) for x in xs[:3]) + extra)
            nv += 1
        for _ in range(int(rng.integers(0, 5))):
            us = rng.random(3)
            third = " " + _obj_num(rng, us[2]) if rng.random() < 0.2 else ""
            out.append("vt\t" + " ".join(_obj_num(rng, u) for u in us[:2]) + third)
            nvt += 1
        for _ in range(int(rng.integers(0, 5))):
            ns = rng.normal(size=3)
            out.append("vn  " + " ".join(_obj_num(rng, n) for n in ns) + "  ")
            nvn += 1
        r = rng.random()
        if r < 0.15:
            name = mats[int(rng.integers(0, len(mats)))]
            out.append("usemtl " + name if rng.random() < 0.9 else "usemtl")
        elif r < 0.2:
            out.append("g part%d" % b)
        elif r < 0.23:
            out.append("o Obj%d" % b)
        for _ in range(int(rng.integers(1, 6))):
            nverts = int(rng.integers(2, 7)) if rng.random() < 0.1 else int(rng.choice([3, 3, 3, 4]))
            form = int(rng.integers(0, 5))
            toks = []
            for _ in range(nverts):
                def ref(count):
                    i = int(rng.integers(0, count))
                    return str(i + 1) if rng.random() < 0.7 else str(i - count)
                v = ref(nv)
                t = ref(nvt) if nvt else ""
                n = ref(nvn) if nvn else ""
                if form == 0 or (form in (1, 3, 4) and not nvt) or (form == 2 and not nvn):
                    toks.append(v)
                elif form == 1:
                    toks.append(v + "/" + t)
                elif form == 2:
                    toks.append(v + "//" + n)
                elif form == 3:
                    toks.append(v + "/" + t + "/" + (n if nvn else ""))
                else:
                    toks.append(v + "/" + t + "/" + (n if nvn else "") + "/9")
            out.append("f " + " ".join(toks))
        if rng.random() < 0.05:
            out.append(["vp 0.5 0.5", "l 1 2", "# café comment", "s 1", "", "   "][int(rng.integers(0, 6))])
    # numbers only the host converts, read as Python's float() does
    out.append("v 1_000.25 inf -nan")
    out.append("v 0.1000000000000000055511151231257827 1e-400 1e400")
    out.append("f -1 -2 -3")
    enders = ["\n"] * 18 + ["\r\n", "\r"]
    return "".join(line + enders[int(rng.integers(0, len(enders)))] for line in out) + "f 1 2 3"


def _tree(node, indexed):
    shapes = []
    for s in node.shapes:
        g = s.geometry
        tris = g.triangle_count if indexed else len(g._triangles)
        shapes.append({"name": s.name if hasattr(s, "name") else "", "groups": sorted(s.material_groups.keys()),
                       "tris": int(tris)})
    return {"name": node.name, "shapes": shapes, "children": [_tree(c, indexed) for c in node.children]}


def make_obj(out_dir):
    """obj_*.npz: OBJ text and what OBJReader (scene/io/obj_reader.py) reads
    from it: load_as_indexed_mesh arrays, _parse_indexed material groups,
    the load(indexed=True / False) hierarchies and the printed warnings."""
    import contextlib
    import io
    import json
    import tempfile
    from scene.io.obj_reader import OBJReader

    cases = {
        "obj_small": ("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvn 0 0 1\n"
                      "usemtl matA\nf 1/1/1 2/2/1 3/3/1\nusemtl matB\nf 2//1 4//1 3//1\nf 1 2 3 4\n"
                      "usemtl matA\nf -4 -3 -2\n"),
        "obj_random": _obj_text(7, 160),
    }
    for name, text in cases.items():
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, name + ".obj")
            with open(path, "w", newline="") as f:
                f.write(text)
            warn = io.StringIO()
            with contextlib.redirect_stdout(warn):
                mesh, mat_groups = OBJReader._parse_indexed(path)
            tree_ix = _tree(OBJReader.load(path, indexed=True), True)
            with contextlib.redirect_stdout(io.StringIO()):
                tree_py = _tree(OBJReader.load(path, indexed=False), False)
        z = lambda a, w: np.zeros((0, w)) if a is None else np.asarray(a)
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"),
            text=np.frombuffer(text.encode("utf-8"), np.uint8),
            positions=z(mesh._positions, 3), normals=z(mesh._normals, 3), uvs=z(mesh._uvs, 2),
            has_normals=mesh._normals is not None, has_uvs=mesh._uvs is not None,
            tri_pos_idx=mesh._tri_pos_idx, tri_normal_idx=mesh._tri_normal_idx, tri_uv_idx=mesh._tri_uv_idx,
            tri_group_idx=mesh._tri_group_idx,
            meta=np.frombuffer(json.dumps({"groups": list(mesh._groups), "mat_groups": sorted(mat_groups),
                                           "tree_indexed": tree_ix, "tree_python": tree_py,
                                           "warnings": warn.getvalue().splitlines()}).encode(), np.uint8))
        print(name + ".npz written", mesh.vertex_count, "verts", mesh.triangle_count, "tris")


def make_rxb(out_dir):
    """meshes.rxb: an archive written by save_rxb_meshes
    (scene/io/roxy_binary.py:13-83), two meshes sharing one position buffer."""
    from scene.io.roxy_binary import save_rxb_meshes
    from scene.mesh import IndexedMesh
    rng = np.random.default_rng(11)
    pos = rng.normal(size=(40, 3))
    a = IndexedMesh(pos, rng.integers(0, 40, size=(25, 3)), normals=rng.normal(size=(40, 3)),
                    tri_normal_idx=rng.integers(0, 40, size=(25, 3)), uvs=rng.random((40, 2)),
                    tri_uv_idx=rng.integers(0, 40, size=(25, 3)), groups=["paint", "rubber"],
                    tri_group_idx=rng.integers(0, 2, size=25), name="frame", build_bvh=False)
    b = IndexedMesh(pos, rng.integers(0, 40, size=(7, 3)), name="wheel", build_bvh=False)
    save_rxb_meshes(os.path.join(out_dir, "meshes.rxb"), {"frame": a, "parts/wheel": b})
    print("meshes.rxb written")


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ROXY_REFERENCE")
    if not ref_root or not os.path.isdir(ref_root):
        raise SystemExit("usage: make_golden.py <reference checkout>")
    _setup(ref_root)
    np.seterr(all="ignore")
    makers = [make_bvh, make_denoise, make_sampling, make_prims, make_traversal, make_trace_scene,
              make_texture_scene, make_obj, make_rxb]
    only = sys.argv[2:]  # optional generator names, e.g. make_texture_scene
    for fn in makers:
        if not only or fn.__name__ in only:
            fn(HERE)


if __name__ == "__main__":
    main()
