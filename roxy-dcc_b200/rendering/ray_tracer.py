"""RayTracer with the reference's signature and validation
(rendering/ray_tracer.py:288-584), rendering through the same GPU wavefront
path as TaichiRenderer.  `threaded` is accepted and ignored (the work is on
the device).  Adaptive sampling stops when the mean absolute change of the
linear accumulator between checks falls to `adaptive_threshold`
(ray_tracer.py:526-541)."""
import math
import time

import numpy as np

import roxy_native as nat
from rendering.render_stats import RenderStats
from rendering.taichi.extractor import build_device_scene
from rendering.taichi.trace import make_params


class RayTracer:
    def __init__(self, world, image, viewport, samples=64, max_depth=8, threaded=True, direct_light_mode="one",
                 denoise=False, denoise_radius=1, denoise_sigma=0.08, denoise_amount=0.8, sample_clamp=10.0,
                 adaptive_sampling=False, adaptive_min_samples=4, adaptive_threshold=0.002,
                 adaptive_check_interval=1, direct_light_max_depth=1, startup_progress=None, *,
                 reference_compat=False, denoise_passes=1, seed=0):
        self._world = world
        self._image = image
        self._viewport = viewport
        self._camera = world.active_camera
        self._samples = samples
        self._max_depth = max_depth
        self._threaded = threaded
        if direct_light_mode not in ("one", "random", "sample", "all", "final"):
            raise ValueError("direct_light_mode must be 'one' or 'all'")
        self._direct_light_mode = "all" if direct_light_mode in ("all", "final") else "one"
        if direct_light_max_depth is None:
            direct_light_max_depth = max_depth
        self._direct_light_max_depth = max(0, int(direct_light_max_depth))
        self._denoise = denoise
        self._denoise_radius = denoise_radius
        self._denoise_sigma = denoise_sigma
        self._denoise_amount = denoise_amount
        self._denoise_passes = int(denoise_passes)
        self._sample_clamp = sample_clamp
        if adaptive_min_samples < 1:
            raise ValueError("adaptive_min_samples must be at least 1")
        if adaptive_threshold < 0:
            raise ValueError("adaptive_threshold must be non-negative")
        if adaptive_check_interval < 1:
            raise ValueError("adaptive_check_interval must be at least 1")
        self._adaptive_sampling = adaptive_sampling
        self._adaptive_min_samples = adaptive_min_samples
        self._adaptive_threshold = adaptive_threshold
        self._adaptive_check_interval = adaptive_check_interval
        self._adaptive_stopped = False
        self._last_adaptive_error = None
        self._last_ray_count = 0
        self._last_stats = None
        self._startup_progress = startup_progress
        self._reference_compat = bool(reference_compat)
        self._seed = int(seed)
        self._accum = None

    def render(self):
        W, H = self._image.width, self._image.height
        start = time.perf_counter()
        self._adaptive_stopped = False
        self._last_adaptive_error = None
        ds = build_device_scene(self._world, method="lbvh")
        ds.use_lights(self._reference_compat)
        if self._accum is None or (self._accum.width, self._accum.height) != (W, H):
            self._accum = nat.Accumulator(W, H)
        acc = self._accum
        acc.reset()
        cam = self._camera
        p = make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, self._max_depth,
                        int(self._world._use_sky), 1 if self._direct_light_mode == "all" else 0,
                        self._direct_light_max_depth, self._sample_clamp, list(self._world._background_color),
                        list(cam.position), list(cam.forward), list(cam.right), list(cam.up),
                        reference_compat=self._reference_compat, seed=self._seed)
        frames = 0
        if not self._adaptive_sampling and not self._viewport:
            if self._samples > 0:
                acc.render(ds.native, p, self._samples)
            frames = self._samples
        else:
            prev = None
            while frames < self._samples:
                acc.render(ds.native, p, 1)
                frames += 1
                if self._viewport:
                    self._image.pixels[:] = acc.read(nat.RX_ACC_DISPLAY)
                    self._viewport.update(self._image)
                    self._viewport.poll_events()
                    if getattr(self._viewport, "should_close", False):
                        break
                if self._adaptive_sampling:
                    cur = acc.read(nat.RX_ACC_RADIANCE)
                    if prev is not None:
                        self._last_adaptive_error = float(np.mean(np.abs(cur - prev)))
                        if (frames < self._samples and frames >= self._adaptive_min_samples and
                                (frames - self._adaptive_min_samples) % self._adaptive_check_interval == 0 and
                                self._last_adaptive_error <= self._adaptive_threshold):
                            self._adaptive_stopped = True
                            prev = cur
                            break
                    prev = cur
        if self._denoise:
            dp = nat.DenoiseParams(int(self._denoise_radius), max(self._denoise_passes, 1), float(self._denoise_sigma),
                                   0.35, 0.20, 1.0, float(self._denoise_amount), 1, 1, 1, 1)
            self._image.pixels[:] = acc.denoise(dp)
        else:
            self._image.pixels[:] = acc.read(nat.RX_ACC_DISPLAY)
        info = acc.info()
        self._last_ray_count = info["rays"]
        self._last_stats = RenderStats(width=W, height=H, samples_requested=self._samples, samples_rendered=frames,
                                       max_depth=self._max_depth, rays_cast=info["rays"],
                                       elapsed_seconds=time.perf_counter() - start,
                                       adaptive_sampling=self._adaptive_sampling,
                                       adaptive_stopped=self._adaptive_stopped,
                                       adaptive_threshold=self._adaptive_threshold,
                                       adaptive_error=self._last_adaptive_error,
                                       adaptive_min_samples=self._adaptive_min_samples)

    @property
    def last_ray_count(self):
        return self._last_ray_count

    @property
    def last_stats(self):
        return self._last_stats

    def __repr__(self):
        return (f"RayTracer(samples={self._samples}, max_depth={self._max_depth}, "
                f"direct_light_mode={self._direct_light_mode!r})")
