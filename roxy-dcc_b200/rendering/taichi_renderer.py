"""TaichiRenderer with the reference's signature
(rendering/taichi_renderer.py:26-203), rendering on the B200 wavefront path.

render(): extract the world to the device (GPU BVH build), run `samples`
progressive frames (CUDA-graph replayed wavefronts), optionally denoise the
resident accumulators (edge-aware a-trous; one pass = the reference's
filter) and write display-space pixels into `image.pixels`.

Extra keyword-only options (defaults keep the reference's behaviour where it
is well defined):
  reference_compat  sphere-light-only NEE with emission counted again on
                    BSDF hits, exactly as trace.py; default False samples
                    emissive triangles and spheres without double counting
  denoise_passes    a-trous passes (1 = the reference's single filter)
  seed              key of the counter-based RNG
  bvh_method        "lbvh" (SAH-collapsed LBVH) or "morton" (reference tree)
  wave_paths        paths per wavefront (0 = automatic)

Unlike the reference, rays are always counted (the counter is free on the
GPU), so `last_ray_count` does not depend on core.timing.LEVEL.
"""
import math
import time

import numpy as np

import roxy_native as nat
from rendering.render_stats import RenderStats
from rendering.taichi import fields
from rendering.taichi.extractor import build_device_scene
from rendering.taichi.trace import make_params


class TaichiRenderer:
    def __init__(self, world, image, viewport, samples=16, max_depth=4, direct_light_mode="one", denoise=False,
                 denoise_radius=1, denoise_sigma=0.08, denoise_amount=0.8, sample_clamp=10.0,
                 direct_light_max_depth=1, startup_progress=None, *, reference_compat=False, denoise_passes=1,
                 seed=0, bvh_method="lbvh", wave_paths=0):
        self._world = world
        self._image = image
        self._viewport = viewport
        self._samples = samples
        self._max_depth = max_depth
        self._direct_light_mode = direct_light_mode
        self._direct_light_mode_id = self._direct_light_mode_to_id(direct_light_mode)
        if direct_light_max_depth is None:
            direct_light_max_depth = max_depth
        self._direct_light_max_depth = max(0, int(direct_light_max_depth))
        self._denoise = denoise
        self._denoise_radius = denoise_radius
        self._denoise_sigma = denoise_sigma
        self._denoise_amount = denoise_amount
        self._denoise_passes = int(denoise_passes)
        self._sample_clamp = sample_clamp
        self._camera = world.active_camera
        self._last_ray_count = 0
        self._last_stats = None
        self._startup_progress = startup_progress
        self._reference_compat = bool(reference_compat)
        self._seed = int(seed)
        self._bvh_method = bvh_method
        self._wave_paths = int(wave_paths)
        self._accum = None
        self._scene = None

    @staticmethod
    def _direct_light_mode_to_id(mode):
        if mode in (0, "one", "random", "sample"):
            return 0
        if mode in (1, "all", "final"):
            return 1
        raise ValueError("direct_light_mode must be 'one' or 'all'")

    def _params(self, W, H):
        cam = self._camera
        world = self._world
        return make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, self._max_depth,
                           int(world._use_sky), self._direct_light_mode_id, self._direct_light_max_depth,
                           self._sample_clamp, list(world._background_color), list(cam.position),
                           list(cam.forward), list(cam.right), list(cam.up), reference_compat=self._reference_compat,
                           seed=self._seed, wave_paths=self._wave_paths)

    def _copy_display(self, acc, apply_denoise):
        if apply_denoise and self._denoise:
            p = nat.DenoiseParams(int(self._denoise_radius), max(self._denoise_passes, 1),
                                  float(self._denoise_sigma), 0.35, 0.20, 1.0, float(self._denoise_amount), 1, 1, 1,
                                  1)
            self._image.pixels[:] = acc.denoise(p)
        else:
            px = self._image.pixels
            if px.dtype == np.float32 and px.flags["C_CONTIGUOUS"]:
                acc.read(nat.RX_ACC_DISPLAY, out=px)  # straight into the image
            else:
                px[:] = acc.read(nat.RX_ACC_DISPLAY)

    def render(self):
        W, H = self._image.width, self._image.height
        start = time.perf_counter()
        if self._startup_progress:
            self._startup_progress.step("Extracting scene for GPU", "Flattening objects, materials and lights.")
        ds = build_device_scene(self._world, method=self._bvh_method)
        fields.bind_scene(ds)
        ds.use_lights(self._reference_compat)
        self._scene = ds
        if self._accum is None or (self._accum.width, self._accum.height) != (W, H):
            self._accum = nat.Accumulator(W, H)
        acc = self._accum
        acc.reset()
        params = self._params(W, H)
        if self._startup_progress:
            self._startup_progress.close()
            self._startup_progress = None
        frames = 0
        if self._viewport and self._samples > 0:
            acc.render(ds.native, params, 1)
            frames = 1
            self._copy_display(acc, False)
            self._viewport.update(self._image)
            self._viewport.poll_events()
            while frames < self._samples and not getattr(self._viewport, "should_close", False):
                k = min(4, self._samples - frames)
                acc.render(ds.native, params, k)
                frames += k
                self._copy_display(acc, False)
                self._viewport.update(self._image)
                self._viewport.poll_events()
        elif self._samples > 0:
            acc.render(ds.native, params, self._samples)
            frames = self._samples
        self._copy_display(acc, True)
        info = acc.info()
        self._last_ray_count = info["rays"]
        st = ds.stats
        self._last_stats = RenderStats(width=W, height=H, samples_requested=self._samples, samples_rendered=frames,
                                       max_depth=self._max_depth, rays_cast=info["rays"],
                                       elapsed_seconds=time.perf_counter() - start,
                                       primitive_count=st.get("primitive_count", 0), bvh_nodes=st.get("bvh_nodes", 0),
                                       bvh_triangles=st.get("bvh_triangles", 0),
                                       bvh_materials=st.get("bvh_materials", 0),
                                       bvh_leaf_size=st.get("bvh_leaf_size", 0))

    @property
    def accumulator(self):
        return self._accum

    @property
    def last_ray_count(self):
        return self._last_ray_count

    @property
    def last_stats(self):
        return self._last_stats

    def __repr__(self):
        return (f"TaichiRenderer(samples={self._samples}, max_depth={self._max_depth}, "
                f"direct_light_mode={self._direct_light_mode!r})")
