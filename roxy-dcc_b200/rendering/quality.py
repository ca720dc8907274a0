"""Image error against high-spp reference renders.

relMSE = mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2), the
reference being a float64-accumulated render of the same scene with the
same sample clamp and an independent random seed.
"""
import ctypes

import numpy as np

import roxy_native as nat


def rel_mse(x, ref, eps=1e-2):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if x.shape != ref.shape:
        raise ValueError(f"image shapes differ: {x.shape} vs {ref.shape}")
    return float(np.mean((x - ref) ** 2 / (ref * ref + eps)))


def reference_render(native_scene, params, spp, seed=0x5EED5EED, ctx=None):
    """float64 mean radiance (H, W, 3) of an `spp`-sample render of
    `native_scene` with `params` (rx_render_params) under another seed."""
    p = type(params).from_buffer_copy(params)
    p.seed = ctypes.c_uint32(seed).value
    acc = nat.Accumulator(p.width, p.height, ctx)
    try:
        acc.set_f64(True)
        acc.render(native_scene, p, int(spp))
        return acc.read_f64()
    finally:
        acc.close()
