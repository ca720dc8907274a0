"""Wavefront renderer parity.

1. Same random numbers: the CUDA wavefront and the oracle's per-path loop
   draw identical Philox numbers, so per-pixel radiance agrees closely
   (differences come only from sin/cos/acos last bits that can send a
   grazing path elsewhere).
2. Statistical: the default estimator (NEE to emissive triangles and
   spheres) converges to the reference estimator (reference_compat, sphere
   lights only, as trace.py): per-pixel means agree within 3 sigma.
3. Ray-count and guide contracts of the reference renderers.
"""
import math

import numpy as np
import pytest

import golden_scenes as gs
import helpers
import roxy_native as nat
import workloads
from oracle import oracle
from rendering.image import Image
from rendering.ray_tracer import RayTracer
from rendering.taichi.extractor import HostScene, build_device_scene
from rendering.taichi.trace import make_params
from rendering.taichi_renderer import TaichiRenderer
from test_host_logic import _ns

pytestmark = pytest.mark.gpu


def _gpu_render(world, W, H, spp, max_depth, compat=False, mode=0, dlmd=1, clamp=10.0, seed=0, wave_paths=0,
                method="lbvh"):
    ds = build_device_scene(world, method=method)
    ds.use_lights(compat)
    cam = world.active_camera
    p = make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, max_depth, world._use_sky, mode,
                    dlmd, clamp, list(world._background_color), list(cam.position), list(cam.forward),
                    list(cam.right), list(cam.up), reference_compat=compat, seed=seed, wave_paths=wave_paths)
    acc = nat.Accumulator(W, H)
    acc.render(ds.native, p, spp)
    out = {k: acc.read(w) for k, w in (("radiance", nat.RX_ACC_RADIANCE), ("normal", nat.RX_ACC_NORMAL),
                                       ("albedo", nat.RX_ACC_ALBEDO), ("depth", nat.RX_ACC_DEPTH),
                                       ("pixels", nat.RX_ACC_DISPLAY))}
    out["rays"] = acc.info()["rays"]
    return out


def _oracle_render(world, W, H, spp, max_depth, compat=False, mode=0, dlmd=1, clamp=10.0, seed=0):
    h = HostScene(world)
    sc = helpers.oracle_scene(h, compat)
    p = helpers.oracle_params(world, W, H, max_depth, compat=compat, mode=mode, dlmd=dlmd, clamp=clamp, seed=seed)
    return oracle.render(sc, p, spp)


def _agree(a, b, tol=1e-4):
    d = np.abs(a - b) / (np.abs(b) + 1e-2)
    return float(np.mean(np.all(d < tol, axis=-1) if d.ndim == 3 else d < tol))


@pytest.mark.parametrize("compat,mode,dlmd", [(False, 0, 8), (True, 0, 8), (False, 1, 2), (True, 1, 1)])
def test_trace_scene_same_randoms_as_oracle(compat, mode, dlmd):
    world = gs.build_trace_scene(_ns())
    W = H = 48
    g = _gpu_render(world, W, H, 6, 8, compat, mode, dlmd, seed=3)
    o = _oracle_render(world, W, H, 6, 8, compat, mode, dlmd, seed=3)
    assert _agree(g["radiance"], o["radiance"]) > 0.97
    assert abs(g["radiance"].mean() - o["radiance"].mean()) < 0.01 * o["radiance"].mean() + 1e-4
    assert abs(g["rays"] - o["rays"]) <= 0.01 * o["rays"]
    # first-hit guides and display buffer
    assert _agree(g["normal"], o["normal"], 1e-3) > 0.97
    assert _agree(g["albedo"], o["albedo"], 1e-4) > 0.97
    assert _agree(g["depth"], o["depth"], 1e-4) > 0.97
    assert _agree(g["pixels"], o["pixels"], 1e-3) > 0.97


@pytest.mark.parametrize("indexed,method,compat", [(False, "lbvh", False), (True, "lbvh", True),
                                                   (True, "morton", False), (False, "morton", True)])
def test_textured_scene_same_randoms_as_oracle(indexed, method, compat):
    """Texture-mapped albedo (trace.py:96-136) on both extraction paths: the
    radiance and first-hit albedo guide follow the oracle pixel by pixel."""
    world = gs.build_texture_scene(_ns(), indexed=indexed)
    W = H = 48
    g = _gpu_render(world, W, H, 6, 6, compat, 0, 2, seed=5, method=method)
    o = _oracle_render(world, W, H, 6, 6, compat, 0, 2, seed=5)
    assert _agree(g["radiance"], o["radiance"]) > 0.97
    assert _agree(g["albedo"], o["albedo"], 1e-5) > 0.99
    assert abs(g["rays"] - o["rays"]) <= 0.01 * o["rays"]
    # the textures are really sampled: the first-hit albedo varies across a
    # single-material textured face
    assert np.unique(np.round(g["albedo"][H // 4:H // 2, W // 4:W // 2, 0], 4)).size > 4


def test_cornell_same_randoms_and_wavefront_sizes():
    world = workloads.cornell_box(64, 64)
    o = _oracle_render(world, 64, 64, 8, 8, dlmd=8, seed=1)
    for wp in (0, 4096, 64 * 64 * 3):
        g = _gpu_render(world, 64, 64, 8, 8, dlmd=8, seed=1, wave_paths=wp)
        assert _agree(g["radiance"], o["radiance"]) > 0.98, wp
        assert abs(g["rays"] - o["rays"]) <= 0.005 * o["rays"]


def _batch_means(world, W, H, batches, per, compat, seed0, dlmd=8, max_depth=8, mis=False, mode=0):
    ds = build_device_scene(world, method="lbvh")
    ds.use_lights(compat)
    cam = world.active_camera
    acc = nat.Accumulator(W, H)
    means = []
    for b in range(batches):
        acc.reset()
        p = make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, max_depth, world._use_sky,
                        mode, dlmd, 0.0, list(world._background_color), list(cam.position), list(cam.forward),
                        list(cam.right), list(cam.up), reference_compat=compat, seed=seed0 + b, mis=mis)
        acc.render(ds.native, p, per)
        means.append(acc.read(nat.RX_ACC_RADIANCE))
    return np.array(means)


@pytest.mark.parametrize("scene_name", ["cornell", "trace"])
def test_converges_to_reference_estimator_3sigma(scene_name):
    """Default estimator vs the reference's estimator, unclamped.

    Cornell (light 2 cm under the ceiling): NEE to the emissive quad vs the
    reference's BSDF-only transport (its NEE sees no triangle lights).  Mixed
    scene (sphere light, glass, metal, glossy, plane, cube): NEE vs the
    reference estimator without its sphere-light NEE, whose double count
    makes it converge to a different image by construction.
    Per 2x2 pixel block the means must agree within 3 sigma except for a few
    blocks, and the image means within 4 sigma."""
    W = H = 24
    if scene_name == "cornell":
        world = workloads.cornell_box(W, H, light_gap=0.02)
        new = _batch_means(world, W, H, 32, 32, False, 100)
        ref = _batch_means(world, W, H, 32, 32, True, 50000)
    else:
        world = gs.build_trace_scene(_ns())
        new = _batch_means(world, W, H, 32, 32, False, 100)
        ref = _batch_means(world, W, H, 32, 32, True, 50000, dlmd=0)
    n = len(new)
    A = new.reshape(n, H // 2, 2, W // 2, 2, 3).mean((2, 4))
    R = ref.reshape(n, H // 2, 2, W // 2, 2, 3).mean((2, 4))
    se = np.sqrt(A.var(0, ddof=1) / n + R.var(0, ddof=1) / n) + 1e-6
    z = np.abs(A.mean(0) - R.mean(0)) / se
    assert np.mean(z > 3) < 0.05, np.mean(z > 3)
    ma, mr = new.mean((1, 2, 3)), ref.mean((1, 2, 3))
    zm = abs(ma.mean() - mr.mean()) / np.sqrt(ma.var(ddof=1) / n + mr.var(ddof=1) / n)
    assert zm < 4, (zm, ma.mean(), mr.mean())


def _renders_with_tail(world, W, H, spp, max_depth, dlmd, tails, mode=0, compat=False, mis=False, method="lbvh",
                       wave_paths=0):
    ds = build_device_scene(world, method=method)
    ds.use_lights(compat)
    cam = world.active_camera
    p = make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, max_depth, world._use_sky, mode,
                    dlmd, 10.0, list(world._background_color), list(cam.position), list(cam.forward),
                    list(cam.right), list(cam.up), reference_compat=compat, seed=11, wave_paths=wave_paths)
    if mis:
        p.mis = 1
    outs = []
    for t in tails:
        acc = nat.Accumulator(W, H)
        acc.set_tail(t)
        acc.render(ds.native, p, spp)
        acc.render(ds.native, p, 2)  # a second call continues the running means
        out = [acc.read(w) for w in (nat.RX_ACC_RADIANCE, nat.RX_ACC_NORMAL, nat.RX_ACC_ALBEDO, nat.RX_ACC_DEPTH,
                                     nat.RX_ACC_DISPLAY)]
        outs.append((out, acc.info()["rays"]))
    return outs


@pytest.mark.parametrize("case", ["trace-one", "trace-all", "trace-compat", "trace-reference-tree", "cornell",
                                  "cornell-mis", "cornell-waves", "texture", "icosphere"])
def test_wave_tail_equals_one_launch_per_bounce(case):
    """k_tail (a wave's remaining bounces run path by path in one launch, the
    shadow rays traced at once) gives the same radiance, guides, display and
    ray count bit for bit as one extend and one shade launch per bounce,
    whether it takes over at bounce 1 (threshold above every queue) or part
    way through the wave (threshold between the queue lengths)."""
    W, H, spp = 40, 30, 6
    paths = W * H * spp
    tails = (0, 1 << 30, paths // 9)
    kw = {}
    if case.startswith("trace"):
        world = gs.build_trace_scene(_ns())
        kw = {"trace-one": dict(mode=0), "trace-all": dict(mode=1), "trace-compat": dict(compat=True),
              "trace-reference-tree": dict(method="morton")}[case]
        max_depth, dlmd = 8, 8
    elif case.startswith("cornell"):
        world = workloads.cornell_box(W, H)
        kw = {"cornell": {}, "cornell-mis": dict(mis=True), "cornell-waves": dict(wave_paths=2 * W * H)}[case]
        max_depth, dlmd = 8, 8
    elif case == "texture":
        world = gs.build_texture_scene(_ns())
        max_depth, dlmd = 6, 6
    else:
        world = workloads.displaced_icosphere_scene(W, H, subdiv=4)
        max_depth, dlmd = 12, 1
    outs = _renders_with_tail(world, W, H, spp, max_depth, dlmd, tails, **kw)
    (ref, rays) = outs[0]
    assert rays > paths
    for t, (out, r) in zip(tails[1:], outs[1:]):
        assert r == rays, (t, r, rays)
        for k, (a, b) in enumerate(zip(out, ref)):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (t, k, float(np.abs(a - b).max()))


def _block_z(A, B):
    n = len(A)
    H, W = A.shape[1:3]
    A = A.reshape(n, H // 2, 2, W // 2, 2, 3).mean((2, 4))
    B = B.reshape(len(B), H // 2, 2, W // 2, 2, 3).mean((2, 4))
    se = np.sqrt(A.var(0, ddof=1) / len(A) + B.var(0, ddof=1) / len(B)) + 1e-6
    return np.abs(A.mean(0) - B.mean(0)) / se


@pytest.mark.parametrize("scene_name,mode", [("cornell", 0), ("trace", 0), ("trace", 1)])
def test_mis_converges_to_the_same_image_3sigma(scene_name, mode):
    """Power-heuristic MIS between NEE and BSDF hits of listed lights
    (rendering/sampling.py:36-45) converges to the BSDF-only transport (the
    reference estimator without NEE): the same image within 3 sigma per 2x2
    block.  On the Cornell box, whose light hangs 2 cm under the ceiling
    (NEE alone is heavy-tailed at the ceiling beside it), MIS has a fraction
    of the variance of either strategy alone (measured ~1/29 of NEE's and
    ~1/5 of BSDF-only's)."""
    W = H = 24
    if scene_name == "cornell":
        world = workloads.cornell_box(W, H, light_gap=0.02)
    else:
        world = gs.build_trace_scene(_ns())
    mis = _batch_means(world, W, H, 40, 64, False, 300, mis=True, mode=mode)
    ref = _batch_means(world, W, H, 40, 64, True, 700, dlmd=0)
    z = _block_z(mis, ref)
    assert np.mean(z > 3) < 0.05, np.mean(z > 3)
    ma, mr = mis.mean((1, 2, 3)), ref.mean((1, 2, 3))
    zm = abs(ma.mean() - mr.mean()) / np.sqrt(ma.var(ddof=1) / len(ma) + mr.var(ddof=1) / len(mr))
    assert zm < 4, (zm, ma.mean(), mr.mean())
    if scene_name == "cornell":
        nee = _batch_means(world, W, H, 40, 64, False, 900, mode=mode)
        assert mis.var(0).mean() < 0.5 * nee.var(0).mean(), (mis.var(0).mean(), nee.var(0).mean())
        assert mis.var(0).mean() < 0.5 * ref.var(0).mean(), (mis.var(0).mean(), ref.var(0).mean())


def _tiny_world(use_sky):
    from core import Color, Vec3
    from scene import Camera, World
    w = World(use_sky=use_sky)
    w.add_camera(Camera(width=4, height=4))
    return w, Vec3, Color


def test_ray_count_contracts():
    w, Vec3, Color = _tiny_world(True)
    rt = RayTracer(w, Image(4, 4), None, samples=3, max_depth=4, threaded=False)
    rt.render()
    assert rt.last_ray_count == 4 * 4 * 3 and rt.last_stats.rays_per_pixel == 3
    assert rt.last_stats.samples_rendered == 3
    assert (Image(4, 4).pixels == 0).all()
    rt = RayTracer(w, Image(4, 4), None, samples=2, max_depth=0, threaded=False)
    rt.render()
    assert rt.last_ray_count == 0 and rt.last_stats.max_depth == 0
    w2, _, _ = _tiny_world(False)
    img = Image(4, 4)
    rt = RayTracer(w2, img, None, samples=1, max_depth=4, threaded=False)
    rt.render()
    assert np.allclose(img.pixels, 0)
    img = Image(4, 4)
    rt = RayTracer(w, img, None, samples=1, max_depth=4, threaded=False)
    rt.render()
    assert img.pixels.max() > 0
    assert "Render report" in rt.last_stats.format_report()


def test_direct_light_depth_zero_skips_shadow_rays():
    from core import Color, Vec3
    from scene import Camera, Diffuse, Emissive, SceneObject, Sphere, World
    w = World(use_sky=False)
    w.add_camera(Camera(width=4, height=4))
    w.add_object(SceneObject(shape=Sphere(), material=Diffuse(Color(0.8, 0.8, 0.8)), translation=Vec3(0, 0, -3)))
    w.add_object(SceneObject(shape=Sphere(), material=Emissive(Color(1, 1, 1), intensity=40.0),
                             translation=Vec3(0, 2, -1), scale=Vec3(0.5, 0.5, 0.5)))
    img = Image(4, 4)
    rt = RayTracer(w, img, None, samples=1, max_depth=1, threaded=False, direct_light_max_depth=0)
    rt.render()
    assert np.allclose(img.pixels, 0) and rt.last_ray_count == 16
    img = Image(4, 4)
    rt = RayTracer(w, img, None, samples=1, max_depth=1, threaded=False)
    rt.render()
    assert img.pixels.sum() > 0 and rt.last_ray_count > 16


def test_taichi_renderer_end_to_end_with_denoise():
    world = workloads.cornell_box(64, 64)
    img = Image(64, 64)
    r = TaichiRenderer(world, img, None, samples=8, max_depth=8, denoise=True, denoise_passes=5,
                       direct_light_max_depth=8)
    r.render()
    s = r.last_stats
    assert s.samples_rendered == 8 and s.rays_cast == r.last_ray_count > 64 * 64 * 8
    assert s.bvh_triangles == 36 and s.bvh_nodes > 0
    assert np.isfinite(img.pixels).all() and 0.05 < img.pixels.mean() < 1.0
    assert img.pixels.max() <= 1.0 and img.pixels.min() >= 0.0
    # the renderer's denoise equals the standalone filter on the same buffers
    acc = r.accumulator
    lin = acc.read(nat.RX_ACC_RADIANCE)
    from rendering.denoise import edge_aware_denoise, linear_to_display
    ref = linear_to_display(edge_aware_denoise(lin, 1, 0.08, 0.8, normal=acc.read(nat.RX_ACC_NORMAL),
                                               albedo=acc.read(nat.RX_ACC_ALBEDO), depth=acc.read(nat.RX_ACC_DEPTH),
                                               passes=5))
    np.testing.assert_allclose(img.pixels, ref, atol=1e-6)


def test_progressive_accumulation_equals_one_shot():
    world = workloads.cornell_box(32, 32)
    ds = build_device_scene(world)
    ds.use_lights(False)
    cam = world.active_camera
    p = make_params(32, 32, math.tan(math.radians(cam.fov) / 2), 1.0, 8, 0, 0, 8, 10.0, [0, 0, 0],
                    list(cam.position), list(cam.forward), list(cam.right), list(cam.up), seed=5)
    a = nat.Accumulator(32, 32)
    a.render(ds.native, p, 12)
    b = nat.Accumulator(32, 32)
    for k in (1, 4, 3, 4):
        b.render(ds.native, p, k)
    np.testing.assert_array_equal(a.read(nat.RX_ACC_RADIANCE), b.read(nat.RX_ACC_RADIANCE))
    assert a.info()["rays"] == b.info()["rays"] and b.info()["frames"] == 12


def test_async_frames_equal_synchronous_frames():
    """An asynchronous accumulator queues reset + render without waiting;
    after a context sync its running means and ray count are bit-identical
    to the synchronous ones, resets included."""
    world = workloads.cornell_box(48, 32)
    ds = build_device_scene(world)
    ds.use_lights(False)
    cam = world.active_camera
    p = make_params(48, 32, math.tan(math.radians(cam.fov) / 2), 1.5, 8, 0, 0, 8, 10.0, [0, 0, 0],
                    list(cam.position), list(cam.forward), list(cam.right), list(cam.up), seed=3)
    a = nat.Accumulator(48, 32)
    a.render(ds.native, p, 8)
    b = nat.Accumulator(48, 32)
    b.set_async(True)
    b.render(ds.native, p, 5)
    b.reset()
    for k in (3, 5):
        b.render(ds.native, p, k)
    b.ctx.sync()
    b.set_async(False)
    np.testing.assert_array_equal(a.read(nat.RX_ACC_RADIANCE), b.read(nat.RX_ACC_RADIANCE))
    np.testing.assert_array_equal(a.read(nat.RX_ACC_DISPLAY), b.read(nat.RX_ACC_DISPLAY))
    assert a.info()["rays"] == b.info()["rays"] and b.info()["frames"] == 8
    # a read into a caller's buffer (the renderer reads into its Image)
    out = np.full((32, 48, 3), -1.0, np.float32)
    assert b.read(nat.RX_ACC_DISPLAY, out=out) is out
    np.testing.assert_array_equal(out, a.read(nat.RX_ACC_DISPLAY))
    with pytest.raises(ValueError, match="C-contiguous float32"):
        b.read(nat.RX_ACC_DISPLAY, out=np.zeros((32, 48, 3), np.float64))


def test_reused_accumulator_across_scenes_and_parameters():
    """One accumulator alternating between two scenes and two seeds (its
    wave graph is updated in place with the new arguments) gives the same
    images as fresh accumulators."""
    W = H = 32
    worlds = [workloads.cornell_box(W, H), gs.build_trace_scene(_ns())]
    scenes = []
    for world in worlds:
        ds = build_device_scene(world)
        ds.use_lights(False)
        scenes.append((world, ds))

    def params(world, seed):
        cam = world.active_camera
        return make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, 6, world._use_sky, 0, 6,
                           10.0, list(world._background_color), list(cam.position), list(cam.forward),
                           list(cam.right), list(cam.up), seed=seed)

    shared = nat.Accumulator(W, H)
    for k, (world, ds) in enumerate(scenes * 2):
        p = params(world, 11 + k)
        shared.reset()
        shared.render(ds.native, p, 4)
        fresh = nat.Accumulator(W, H)
        fresh.render(ds.native, p, 4)
        np.testing.assert_array_equal(shared.read(nat.RX_ACC_RADIANCE), fresh.read(nat.RX_ACC_RADIANCE))
        assert shared.info()["rays"] == fresh.info()["rays"]


def test_float64_reference_accumulation_and_relmse():
    """float64 sums agree with the float32 running means, a float64 render
    keeps its f32 outputs unchanged, and relMSE falls roughly as 1/spp."""
    from rendering.quality import reference_render, rel_mse
    world = workloads.cornell_box(64, 64)
    ds = build_device_scene(world)
    ds.use_lights(False)
    cam = world.active_camera
    p = make_params(64, 64, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, 8, world._use_sky, 0, 8, 10.0,
                    list(world._background_color), list(cam.position), list(cam.forward), list(cam.right),
                    list(cam.up), seed=9)
    plain = nat.Accumulator(64, 64)
    plain.render(ds.native, p, 16)
    acc = nat.Accumulator(64, 64)
    acc.set_f64(True)
    acc.render(ds.native, p, 16)
    np.testing.assert_array_equal(acc.read(nat.RX_ACC_RADIANCE), plain.read(nat.RX_ACC_RADIANCE))
    m64 = acc.read_f64()
    np.testing.assert_allclose(m64, acc.read(nat.RX_ACC_RADIANCE), rtol=2e-5, atol=1e-6)
    with pytest.raises(ValueError, match="before the first frame"):
        plain.set_f64(True)
    ref = reference_render(ds.native, p, 1024)
    errs = []
    for spp in (4, 16, 64):
        a = nat.Accumulator(64, 64)
        a.render(ds.native, p, spp)
        errs.append(rel_mse(a.read(nat.RX_ACC_RADIANCE), ref))
    assert errs[0] > errs[1] > errs[2] > 0.0
    assert 2.0 < errs[0] / errs[1] < 8.0 and 2.0 < errs[1] / errs[2] < 8.0


def test_benchmark_scene_same_randoms_as_oracle():
    """The benchmark scene (327,680-triangle displaced icosphere, 64 spheres
    in the LBVH, quad light) at 160 x 90, 2 spp, depth 12, traced by the
    renderer's own launches (camera rays made in bounce 0's extend kernel,
    the 4-wide tree).  First-hit depth and normal guides follow the oracle
    pixel by pixel; radiance as in the other same-randoms tests."""
    world = workloads.displaced_icosphere_scene(160, 90)
    W, H = 160, 90
    g = _gpu_render(world, W, H, 2, 12, dlmd=1, seed=4)
    o = _oracle_render(world, W, H, 2, 12, dlmd=1, seed=4)
    assert _agree(g["depth"], o["depth"], 1e-5) > 0.999
    assert _agree(g["normal"], o["normal"], 1e-4) > 0.995
    assert _agree(g["radiance"], o["radiance"]) > 0.97
    assert abs(g["rays"] - o["rays"]) <= 0.01 * o["rays"]


def test_cornell_configuration_same_randoms_as_oracle():
    """The Cornell-box configuration at its own size: 256 x 256, 16 spp,
    depth 8, NEE at every bounce, against the oracle pixel by pixel with the
    same random numbers (and the ray count the reference would report)."""
    world = workloads.cornell_box()
    g = _gpu_render(world, 256, 256, 16, 8, dlmd=8, seed=2)
    o = _oracle_render(world, 256, 256, 16, 8, dlmd=8, seed=2)
    assert _agree(g["radiance"], o["radiance"]) > 0.97
    assert _agree(g["depth"], o["depth"], 1e-5) > 0.999
    assert abs(g["rays"] - o["rays"]) <= 0.002 * o["rays"]
    assert abs(g["radiance"].mean() - o["radiance"].mean()) < 0.002 * o["radiance"].mean()


def test_benchmark_configuration_quarter_frame_same_randoms_as_oracle():
    """The benchmark scene at a quarter of its frame (960 x 540), 4 spp,
    depth 12: 2.1 M paths through the renderer's own launches against the
    oracle with the same random numbers."""
    world = workloads.displaced_icosphere_scene(960, 540)
    g = _gpu_render(world, 960, 540, 4, 12, dlmd=1, seed=6)
    o = _oracle_render(world, 960, 540, 4, 12, dlmd=1, seed=6)
    assert _agree(g["radiance"], o["radiance"]) > 0.97
    assert _agree(g["depth"], o["depth"], 1e-5) > 0.999
    assert abs(g["rays"] - o["rays"]) <= 0.002 * o["rays"]
