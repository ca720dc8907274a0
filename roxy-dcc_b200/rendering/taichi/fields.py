"""Process-wide render state for the module-level API.

The reference keeps its scene and accumulators in global Taichi fields
(rendering/taichi/fields.py:14-88) that `extract_scene`, `GPUBVHBuilder.upload`
and `render_kernel` share.  Here the same names refer to device-resident
state owned by libroxy_cuda.so: `_frame_count[None]`, `_ray_count[None]` and
`to_numpy()` on the accumulators keep working for callers such as
bench_atomic.py.
"""
import numpy as np

import roxy_native as nat

MAX_W = 1920
MAX_H = 1080

_state = {"scene": None, "accum": None}


def bind_scene(device_scene):
    _state["scene"] = device_scene


def bind_builder(builder):
    from rendering.taichi.extractor import DeviceScene
    stats = {"primitive_count": 0, "bvh_nodes": len(builder.nodes), "bvh_triangles": builder.triangle_count,
             "bvh_materials": len(builder.mat_palette), "bvh_leaf_size": builder.MAX_LEAF_SIZE}
    _state["scene"] = DeviceScene.from_builder(builder, [], stats)


def current_scene():
    return _state["scene"]


def accumulator(width, height):
    acc = _state["accum"]
    if acc is None or acc.width != width or acc.height != height:
        acc = nat.Accumulator(width, height)
        _state["accum"] = acc
    return acc


class _Scalar:
    def __init__(self, getter, setter):
        self._get, self._set = getter, setter

    def __getitem__(self, key):
        return self._get()

    def __setitem__(self, key, value):
        self._set(value)


def _get_frames():
    acc = _state["accum"]
    return 0 if acc is None else acc.info()["frames"]


def _set_frames(v):
    acc = _state["accum"]
    if acc is not None and int(v) == 0:
        acc.reset()


_ray_base = [0]


def _get_rays():
    acc = _state["accum"]
    return 0 if acc is None else acc.info()["rays"] - _ray_base[0]


def _set_rays(v):
    acc = _state["accum"]
    _ray_base[0] = (0 if acc is None else acc.info()["rays"]) - int(v)


_frame_count = _Scalar(_get_frames, _set_frames)
_ray_count = _Scalar(_get_rays, _set_rays)


class _Buffer:
    def __init__(self, which):
        self.which = which

    def to_numpy(self):
        acc = _state["accum"]
        if acc is None:
            shape = (MAX_H, MAX_W) if self.which == nat.RX_ACC_DEPTH else (MAX_H, MAX_W, 3)
            return np.zeros(shape, np.float32)
        return acc.read(self.which)


_pixels = _Buffer(nat.RX_ACC_DISPLAY)
_accumulator = _Buffer(nat.RX_ACC_RADIANCE)
_normal_accumulator = _Buffer(nat.RX_ACC_NORMAL)
_albedo_accumulator = _Buffer(nat.RX_ACC_ALBEDO)
_depth_accumulator = _Buffer(nat.RX_ACC_DEPTH)
