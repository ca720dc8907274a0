"""Batched rendering of many scenes and its autotuner.

The reference renders one world per TaichiRenderer.render() call
(rendering/taichi_renderer.py:87-191), a full launch sequence per frame.
Here a batch of jobs (scene, accumulator, render parameters, frames) is
traced as shared wavefronts: each wave packs frames of several jobs into
one path space, so every bounce is one extend and one shade launch for all
scenes, and all waves of a call replay as one CUDA graph (rx_batch_*).

The autotuner picks the wavefront size, the extend kernel's block shape and
the BVH leaf size by timing a one-frame probe of the batch on scratch
accumulators, and remembers the choice per batch shape.
"""
import itertools
import math
from dataclasses import dataclass, field

import roxy_native as nat
from rendering.taichi.extractor import build_device_scene
from rendering.taichi.trace import make_params

# Wave sizes: the one-frame probe holds fewer paths than these waves, so it
# cannot rank them; larger waves amortise the tail of every extend launch
# (the 1080p 64-spp single-scene frame: 32 M paths 47.6 ms, 128 M 39.9 ms),
# so the default is one size, 128 M paths (~22 GB of wave state), and the
# probe tunes the leaf size and the extend block.
WAVE_CANDIDATES = (1 << 27,)
BLOCK_CANDIDATES = (64, 128, 256)
LEAF_CANDIDATES = (2, 4, 8)


@dataclass
class BatchConfig:
    wave_paths: int = 1 << 27
    extend_block: int = 128
    leaf_size: int = 4


@dataclass
class Job:
    """One render request: a world at a resolution, spp and depth."""
    world: object
    width: int
    height: int
    spp: int
    max_depth: int
    direct_light_mode: int = 0
    direct_light_max_depth: int = 1
    sample_clamp: float = 10.0
    reference_compat: bool = False
    seed: int = 0
    scene: object = None      # DeviceScene
    acc: object = None        # roxy_native.Accumulator
    params: object = None     # roxy_native.RenderParams
    meta: dict = field(default_factory=dict)

    def prepare(self, leaf_size=4, ctx=None):
        if self.scene is None:
            self.scene = build_device_scene(self.world, method="lbvh", leaf_size=leaf_size)
            self.scene.use_lights(self.reference_compat)
            self.meta["leaf"] = leaf_size
        if self.acc is None:
            self.acc = nat.Accumulator(self.width, self.height, ctx)
        cam = self.world.active_camera
        self.params = make_params(self.width, self.height, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio,
                                  self.max_depth, int(self.world._use_sky), self.direct_light_mode,
                                  self.direct_light_max_depth, self.sample_clamp, list(self.world._background_color),
                                  list(cam.position), list(cam.forward), list(cam.right), list(cam.up),
                                  reference_compat=self.reference_compat, seed=self.seed)
        return self

    def rebuild(self, leaf_size):
        if self.meta.get("leaf") != leaf_size:
            self.scene.native.build_bvh(nat.RX_BVH_LBVH_SAH, min(int(leaf_size), 15), True)
            self.meta["leaf"] = leaf_size

    @property
    def paths(self):
        return self.width * self.height * self.spp


def batch_shape_key(jobs):
    """Coarse shape of a batch: job count, log2 of total paths and of total
    triangles.  Batches of one shape share a tuned configuration."""
    paths = sum(j.paths for j in jobs)
    tris = sum(j.scene.stats["bvh_triangles"] for j in jobs)
    return (len(jobs), int(math.log2(max(paths, 1))), int(math.log2(max(tris, 1))))


def choose(candidates, measure, repeats=2):
    """The candidate with the smallest measured time (best of `repeats`)."""
    best, best_t = None, float("inf")
    timings = []
    for c in candidates:
        t = min(measure(c) for _ in range(repeats))
        timings.append((c, t))
        if t < best_t:
            best, best_t = c, t
    return best, timings


class BatchRenderer:
    """Renders a list of Jobs as one batch; `autotune()` picks its config."""

    _tuned = {}

    def __init__(self, jobs, config=None, ctx=None):
        self.ctx = ctx or nat.context()
        self.jobs = list(jobs)
        self.config = config or BatchConfig()
        for j in self.jobs:
            j.prepare(self.config.leaf_size, self.ctx)
        self.batch = nat.Batch(self.ctx)
        self.tuning = None

    def _load(self, batch, accs, frames_of):
        batch.clear()
        for j, acc in zip(self.jobs, accs):
            batch.add(j.scene.native, acc, j.params, frames_of(j))

    def render(self, frames=None):
        """Render every job's spp (or `frames` frames each) into its own
        accumulator; returns the device milliseconds of the call."""
        c = self.config
        for j in self.jobs:
            j.rebuild(c.leaf_size)
        self.batch.set_config(c.wave_paths, c.extend_block)
        self._load(self.batch, [j.acc for j in self.jobs], lambda j: j.spp if frames is None else frames)
        self.batch.render()
        return self.batch.last_stats()["ms"]

    def autotune(self, waves=WAVE_CANDIDATES, blocks=BLOCK_CANDIDATES, leaves=LEAF_CANDIDATES, use_cache=True):
        """Time a one-frame probe of every job for each (leaf, wave, block)
        and keep the fastest.  Probe frames go to scratch accumulators."""
        key = batch_shape_key(self.jobs)
        if use_cache and key in self._tuned:
            self.config = self._tuned[key]
            self.tuning = {"cached": True, "config": self.config}
            return self.config
        scratch = [nat.Accumulator(j.width, j.height, self.ctx) for j in self.jobs]
        probe = nat.Batch(self.ctx)
        results = []
        try:
            best_leaf, best_leaf_t, best_wb = None, float("inf"), None
            for leaf in leaves:
                for j in self.jobs:
                    j.rebuild(leaf)
                self._load(probe, scratch, lambda j: 1)

                def measure(cfg):
                    probe.set_config(*cfg)
                    for a in scratch:
                        a.reset()
                    probe.render()
                    return probe.last_stats()["ms"]

                wb, timings = choose(list(itertools.product(waves, blocks)), measure)
                t = min(tt for _, tt in timings)
                results += [((leaf,) + cfg, tt) for cfg, tt in timings]
                if t < best_leaf_t:
                    best_leaf, best_leaf_t, best_wb = leaf, t, wb
        finally:
            probe.close()
            for a in scratch:
                a.close()
        self.config = BatchConfig(wave_paths=best_wb[0], extend_block=best_wb[1], leaf_size=best_leaf)
        for j in self.jobs:
            j.rebuild(best_leaf)
        self._tuned[key] = self.config
        self.tuning = {"cached": False, "config": self.config, "probe_ms": best_leaf_t,
                       "timings": [{"leaf": c[0], "wave_paths": c[1], "extend_block": c[2], "ms": t}
                                   for c, t in results]}
        return self.config

    def close(self):
        self.batch.close()
