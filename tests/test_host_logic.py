"""Host-side logic of the drop-in API, checked on the CPU: batches, palette
dedupe, scene flattening, light lists, sampling helpers."""
import os

import numpy as np
import pytest

import golden_scenes as gs
from oracle import oracle
from rendering.sampling import (clamp_color_sample, gpu_pixel_sample_offset, mis_power_weight, philox4x32,
                                pixel_sample_offset)
from rendering.taichi.bvh_builder import GPUBVHBuilder, TriangleBatch
from rendering.taichi.extractor import HostScene, slot_arrays
from rendering.taichi.lights import alias_table

GOLD = os.path.join(os.path.dirname(__file__), "golden")


class NS:
    pass


def _ns():
    import core
    import scene
    ns = NS()
    ns.Vec3, ns.Color = core.Vec3, core.Color
    for n in ("World", "Camera", "SceneObject", "Sphere", "Plane", "Cube", "Mesh", "Triangle", "IndexedMesh",
              "Diffuse", "Metal", "Dielectric", "Shape", "Emissive", "Glossy", "ImageTexture"):
        setattr(ns, n, getattr(scene, n))
    return ns


def _tri(x, **kw):
    d = {'v0': [x, 0, 0], 'v1': [x + 1, 0, 0], 'v2': [x, 1, 0], 'n0': [0, 0, 1], 'n1': [0, 0, 1], 'n2': [0, 0, 1],
         'mat_type': 0, 'albedo': [1, 1, 1], 'roughness': 0.0, 'ior': 1.0, 'emission': 0.0}
    d.update(kw)
    return d


def test_triangle_batch_validation():
    with pytest.raises(ValueError, match="same length"):
        TriangleBatch(np.zeros((2, 3)), np.zeros((1, 3)), np.zeros((2, 3)), np.zeros((2, 3)), np.zeros((2, 3)),
                      np.zeros((2, 3)), [0, 0], np.zeros((2, 3)), [0, 0], [1, 1], [0, 0])
    with pytest.raises(ValueError, match="material arrays must match"):
        TriangleBatch(np.zeros((2, 3)), np.zeros((2, 3)), np.zeros((2, 3)), np.zeros((2, 3)), np.zeros((2, 3)),
                      np.zeros((2, 3)), [0], np.zeros((1, 3)), [0], [1], [0])


def test_indexed_batch_keeps_compact_palette():
    arrays = {'v0': [[0, 0, 0], [2, 0, 0], [4, 0, 0]], 'v1': [[1, 0, 0], [3, 0, 0], [5, 0, 0]],
              'v2': [[0, 1, 0], [2, 1, 0], [4, 1, 0]], 'n0': [[0, 0, 1]] * 3, 'n1': [[0, 0, 1]] * 3,
              'n2': [[0, 0, 1]] * 3, 'uv0': [[0, 0]] * 3, 'uv1': [[1, 0]] * 3, 'uv2': [[0, 1]] * 3,
              'has_uv': [1, 1, 1], 'group_idx': [0, 1, 0]}
    mats = {0: {'mat_type': 0, 'albedo': [1, 0, 0], 'roughness': 0, 'ior': 1, 'emission': 0, 'texture_idx': 3},
            1: {'mat_type': 1, 'albedo': [0, 1, 0], 'roughness': 0.25, 'ior': 1, 'emission': 0, 'texture_idx': -1},
            2: {'mat_type': 0, 'albedo': [0, 0, 1], 'roughness': 0, 'ior': 1, 'emission': 0, 'texture_idx': -1}}
    b = TriangleBatch.from_indexed_arrays(arrays, mats)
    assert b.triangle_count == 3 and len(b.mat_palette) == 2 and list(b.mat_idx) == [0, 1, 0]
    assert b.mat_palette[0]['texture_idx'] == 3


def test_palette_dedupe_matches_reference_builder():
    g = np.load(os.path.join(GOLD, "bvh_palette.npz"))
    batch = TriangleBatch.from_dicts([_tri(0), _tri(2, albedo=[0.5, 0.5, 0.5]), _tri(4, mat_type=1, roughness=0.25),
                                      _tri(6)])
    b = GPUBVHBuilder()
    src = b._material_indices(batch)
    assert [m['type'] for m in b.mat_palette] == list(g["palette_type"])
    np.testing.assert_array_equal(np.array([m['albedo'] for m in b.mat_palette], np.float32), g["palette_albedo"])
    # the golden is in BVH order; the dedupe assigns the same ids per triangle
    assert sorted(src.tolist()) == sorted(g["ordered_mat_idx"].tolist())


def test_concat_mixes_palette_and_per_triangle_batches():
    per_tri = TriangleBatch.from_dicts([_tri(0), _tri(2, albedo=[0.5, 0.5, 0.5])])
    arrays = {'v0': [[0, 0, 0]], 'v1': [[1, 0, 0]], 'v2': [[0, 1, 0]], 'n0': [[0, 0, 1]], 'n1': [[0, 0, 1]],
              'n2': [[0, 0, 1]], 'group_idx': [0]}
    pal = TriangleBatch.from_indexed_arrays(arrays, {0: {'mat_type': 1, 'albedo': [0, 1, 0], 'roughness': 0.3,
                                                         'ior': 1, 'emission': 0}})
    cat = TriangleBatch.concat([per_tri, pal])
    assert cat.triangle_count == 3 and cat.mat_idx is not None
    b = GPUBVHBuilder()
    idx = b._material_indices(cat)
    assert [b.mat_palette[i]['type'] for i in idx] == [0, 0, 1]


def test_indexed_mesh_flattening_matches_reference():
    g = np.load(os.path.join(GOLD, "indexed_arrays.npz"))
    obj = gs.build_indexed_object(_ns())
    geo = obj.shapes[0].geometry
    np.testing.assert_allclose(np.array(obj.world_matrix.rows), g["world_matrix"], rtol=0, atol=1e-15)
    arrs = geo.indexed_triangle_arrays(obj.world_matrix, obj.world_inverse_transpose_matrix)
    for k in ("v0", "v1", "v2", "n0", "n1", "n2", "uv0", "uv1", "uv2", "has_uv", "group_idx"):
        np.testing.assert_array_equal(arrs[k], g[k], err_msg=k)


def test_emissive_rows_use_the_device_kernel_order():
    """Light triangles are transformed on the host in the element-wise order
    of k_extract_indexed; on the golden object that equals the reference's
    BLAS transform after rounding to float32."""
    from rendering.taichi.extractor import _indexed_world_positions
    g = np.load(os.path.join(GOLD, "indexed_arrays.npz"))
    obj = gs.build_indexed_object(_ns())
    geo = obj.shapes[0].geometry
    sel = np.arange(0, geo.triangle_count, 3)
    w = _indexed_world_positions(geo, obj.world_matrix, sel)
    for c, k in enumerate(("v0", "v1", "v2")):
        assert np.array_equal(w[:, c].view(np.uint32), g[k][sel].view(np.uint32)), k


def test_trace_scene_flattening_matches_reference_extract():
    """Object slots, palette and BVH-ordered triangles equal extract_scene's."""
    g = np.load(os.path.join(GOLD, "trace_scene.npz"))
    h = HostScene(gs.build_trace_scene(_ns()))
    sa = slot_arrays(h.slots)
    for k in ("type", "mat_type"):
        np.testing.assert_array_equal(sa[k], g[f"obj_{k}"], err_msg=k)
    for k in ("center", "radius", "normal", "offset", "extra", "v0", "v1", "v2", "albedo", "roughness", "ior",
              "emission"):
        np.testing.assert_allclose(sa[k], g[f"obj_{k}"], rtol=1e-6, atol=1e-7, err_msg=k)
    bvh = oracle.bvh_build_morton(h.batch.v0, h.batch.v1, h.batch.v2, 8)
    np.testing.assert_array_equal(bvh["left"], g["left"])
    o = bvh["order"]
    for k in ("v0", "v1", "v2", "n0", "n1", "n2"):
        np.testing.assert_array_equal(getattr(h.batch, k)[o], g[k], err_msg=k)
    np.testing.assert_array_equal(h.mat_idx[o], g["tri_mat"])
    np.testing.assert_array_equal(h.palette[0], g["mat_type"])
    np.testing.assert_array_equal(h.palette[1], g["mat_albedo"])
    lights = h.lights(compat=True)
    np.testing.assert_allclose(lights["p0"], g["light_center"], rtol=1e-6)
    np.testing.assert_allclose(lights["p1"][:, 0], g["light_radius"], rtol=1e-6)


@pytest.mark.parametrize("indexed", [False, True])
def test_texture_scene_flattening_matches_reference_extract(indexed):
    """Texture table (order, u8 pixels, flips), palette texture indices and
    BVH-ordered uvs equal extract_scene's fields."""
    g = np.load(os.path.join(GOLD, "texture_scene_indexed.npz" if indexed else "texture_scene.npz"))
    h = HostScene(gs.build_texture_scene(_ns(), indexed=indexed))
    assert len(h.textures) == len(g["tex_w"])
    for i, im in enumerate(h.textures):
        np.testing.assert_array_equal(im, g[f"tex{i}"])
    np.testing.assert_array_equal(h.tex_flip, g["tex_flip"])
    np.testing.assert_array_equal(h.mat_texture, g["mat_texture"])
    np.testing.assert_array_equal(h.palette[0], g["mat_type"])
    bvh = oracle.bvh_build_morton(h.batch.v0, h.batch.v1, h.batch.v2, 8)
    o = bvh["order"]
    for k in ("v0", "v1", "v2", "n0", "n1", "n2", "uv0", "uv1", "uv2", "has_uv"):
        np.testing.assert_array_equal(getattr(h.batch, k)[o], g[k], err_msg=k)
    np.testing.assert_array_equal(h.mat_idx[o], g["tri_mat"])
    # the textured emitter is not an explicit light
    lights = h.lights(compat=False)
    assert int(np.sum(lights["kind"] == 1)) == 0


def test_texture_table_limits():
    from rendering.taichi.extractor import MAX_TEXTURES, TextureTable
    ns = _ns()
    table = TextureTable()
    mats = [ns.Diffuse(ns.Color(1, 1, 1), albedo_texture=ns.ImageTexture.from_array(np.ones((2, 2, 3))))
            for _ in range(MAX_TEXTURES)]
    assert [table.index(m) for m in mats] == list(range(MAX_TEXTURES))
    assert table.index(mats[3]) == 3 and table.index(ns.Diffuse(ns.Color(1, 1, 1))) == -1
    with pytest.raises(ValueError, match="more than 8 image textures"):
        table.index(ns.Diffuse(ns.Color(1, 1, 1), albedo_texture=ns.ImageTexture.from_array(np.ones((2, 2, 3)))))
    with pytest.raises(ValueError, match="needs either a path or pixel array"):
        ns.ImageTexture()
    with pytest.raises(RuntimeError, match="pygame"):
        ns.ImageTexture(path="x.png").load_pixels_u8()


def test_alias_table_reproduces_distribution():
    w = np.array([1.0, 3.0, 0.5, 5.5, 0.0])
    prob, alias, pdf = alias_table(w)
    n = len(w)
    got = np.zeros(n)
    for c in range(n):
        got[c] += prob[c] / n
        got[alias[c]] += (1 - prob[c]) / n
    np.testing.assert_allclose(got, w / w.sum(), atol=1e-6)
    np.testing.assert_allclose(pdf, w / w.sum(), atol=1e-7)


def test_philox_python_matches_oracle():
    for ctr, key in (([0, 0, 0, 0], (0, 0)), ([1, 2, 3, 4], (5, 6)), ([0xFFFFFFFF] * 4, (7, 0x5EEDC0DE))):
        assert list(philox4x32(ctr, key)) == list(oracle.philox(ctr, *key))


def test_sampling_helpers_match_reference_contracts():
    g = np.load(os.path.join(GOLD, "sampling.npz"))["offsets"]
    for y in range(16):
        for x in range(16):
            for f in range(8):
                assert pixel_sample_offset(x, y, f) == tuple(g[y, x, f])
    for f in range(8):
        jx, jy = gpu_pixel_sample_offset(12, 34, f, 64)
        assert 0.0 <= jx < 1.0 and 0.0 <= jy < 1.0
    assert gpu_pixel_sample_offset(4, 5, 0, 64) != gpu_pixel_sample_offset(4, 5, 1, 64)
    assert gpu_pixel_sample_offset(4, 5, 0, 64) != gpu_pixel_sample_offset(5, 5, 0, 64)
    from core import Color
    c = Color(20, -1, 2)
    assert clamp_color_sample(c, None) is c and clamp_color_sample(c, 0) is c
    cc = clamp_color_sample(c, 10.0)
    assert (cc.r, cc.g, cc.b) == (10.0, 0.0, 2.0)
    assert abs(mis_power_weight(2.0, 2.0) - 0.5) < 1e-12
    assert mis_power_weight(0.0, 4.0) == 0.0 and mis_power_weight(4.0, 0.0) == 1.0 and mis_power_weight(0, 0) == 0


def test_renderer_rejects_bad_light_mode():
    from rendering.image import Image
    from rendering.ray_tracer import RayTracer
    from rendering.taichi_renderer import TaichiRenderer
    import workloads
    w = workloads.cornell_box(8, 8)
    with pytest.raises(ValueError):
        TaichiRenderer(w, Image(8, 8), None, direct_light_mode="bogus")
    with pytest.raises(ValueError):
        RayTracer(w, Image(8, 8), None, direct_light_mode="bogus")
    with pytest.raises(ValueError):
        RayTracer(w, Image(8, 8), None, adaptive_min_samples=0)
    assert "3" in repr(TaichiRenderer(w, Image(8, 8), None, samples=3))


def test_autotuner_choice_and_batch_specs():
    import workloads
    from rendering.batch import choose
    calls = []

    def measure(c):
        calls.append(c)
        return {(1, 64): 3.0, (1, 128): 2.0, (2, 64): 2.5, (2, 128): 4.0}[c]

    best, timings = choose([(1, 64), (1, 128), (2, 64), (2, 128)], measure, repeats=2)
    assert best == (1, 128) and len(calls) == 8 and len(timings) == 4
    specs = workloads.batch_specs()
    assert len(specs) == 64
    tris = np.array([s["n_tris"] for s in specs])
    assert tris.min() >= 1000 and tris.max() <= 2_000_000 and 10e6 < tris.sum() < 30e6
    assert {s["width"] for s in specs} <= {256, 512, 1024} and {s["spp"] for s in specs} <= {1, 4, 16, 64}
    assert all(4 <= s["max_depth"] <= 16 for s in specs)
    assert specs == workloads.batch_specs()  # seeded


def test_rel_mse_definition():
    from rendering.quality import rel_mse
    ref = np.array([[[0.0, 1.0, 2.0]]])
    x = np.array([[[0.1, 1.0, 1.0]]])
    want = np.mean([0.01 / 0.01, 0.0, 1.0 / 4.01])
    assert abs(rel_mse(x, ref) - want) < 1e-12
    assert rel_mse(ref, ref) == 0.0
    with pytest.raises(ValueError):
        rel_mse(np.zeros((2, 2, 3)), np.zeros((2, 3, 3)))


def test_running_mean_quotient_equals_ieee_division():
    """k_accumulate divides every channel of a frame's running mean by
    d = frame + 1 as RN(x * RN(1/d)) plus one FMA correction step
    (Markstein's), returning RN(x * RN(1/d)) itself when the residual is
    zero; within the range where the kernel uses it (zeros included), that
    is the correctly rounded quotient, the same float as x / d.  Checked with the
    same IEEE operations on the host (libm fmaf), over random floats of the
    accumulators' magnitudes and frame counts up to 2^16."""
    import ctypes
    import ctypes.util
    libm = ctypes.CDLL(ctypes.util.find_library("m"))
    libm.fmaf.restype = ctypes.c_float
    libm.fmaf.argtypes = [ctypes.c_float] * 3
    rng = np.random.default_rng(12)
    f32 = np.float32
    d_all = np.concatenate([np.arange(2, 200), rng.integers(200, 1 << 16, 300)]).astype(np.float32)
    mags = np.float32(10.0) ** rng.uniform(-28, 28, 40000).astype(np.float32)
    xs = (mags * rng.choice([-1, 1], 40000)).astype(np.float32)
    xs[:4] = [0.0, -0.0, 1.0, -0.5]
    bad = 0
    for k, x in enumerate(xs):
        d = d_all[k % len(d_all)]
        r = f32(1.0) / d
        q = f32(x * r)
        res = f32(libm.fmaf(-q, d, x))
        got = q if res == 0.0 else f32(libm.fmaf(res, r, q))
        bad += int(got.view(np.uint32) != f32(x / d).view(np.uint32))
    assert bad == 0
