"""Test helpers: turn a world into the oracle's reference-layout scene.

The oracle gets the same flattened triangles, palette, object slots and
light lists as the CUDA path, with its own (reference) Morton BVH.
"""
import numpy as np

from oracle import oracle


def oracle_scene(host, compat):
    """host: rendering.taichi.extractor.HostScene."""
    b = host.batch
    kw = {}
    if b.triangle_count:
        bvh = oracle.bvh_build_morton(b.v0, b.v1, b.v2, 8)
        o = bvh["order"]
        kw = dict(node_min=bvh["node_min"], node_max=bvh["node_max"], left=bvh["left"], right=bvh["right"],
                  start=bvh["start"], count=bvh["count"], v0=b.v0[o], v1=b.v1[o], v2=b.v2[o], n0=b.n0[o],
                  n1=b.n1[o], n2=b.n2[o], tri_mat=host.mat_idx[o])
        if host.textures:
            kw.update(uv0=b.uv0[o], uv1=b.uv1[o], uv2=b.uv2[o], has_uv=b.has_uv[o], mat_texture=host.mat_texture,
                      textures=host.textures, tex_flip=host.tex_flip)
    pt, pa, pr, pi, pe = host.palette
    objects = None
    if host.slots:
        from rendering.taichi.extractor import slot_arrays
        objects = slot_arrays(host.slots)
    lights = host.lights(compat)
    if lights is not None:
        lights = dict(lights)
        lights["obj"] = np.zeros(len(lights["kind"]), np.int32)
    return oracle.Scene(mat_type=pt, mat_albedo=pa, mat_roughness=pr, mat_ior=pi, mat_emission=pe,
                        objects=objects, lights=lights, **kw)


def oracle_params(world, width, height, max_depth, compat=False, mode=0, dlmd=1, clamp=10.0, seed=0):
    import math
    cam = world.active_camera
    return oracle.make_params(width, height, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio,
                              list(cam.position), list(cam.forward), list(cam.right), list(cam.up), max_depth,
                              int(world._use_sky), list(world._background_color), direct_light_mode=mode,
                              direct_light_max_depth=dlmd, sample_clamp=clamp, reference_compat=int(compat),
                              seed=seed)
