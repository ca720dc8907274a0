"""Edge-aware denoise (rendering/denoise.py API) on the GPU.

`edge_aware_denoise` runs the reference's guided bilateral filter as pass 0
of the CUDA a-trous kernel (`passes=1`); more passes dilate the taps 2^i.
"""
import numpy as np

import roxy_native as nat


def _guide(name, guide, shape, channels):
    if guide is None:
        return None
    arr = np.asarray(guide, dtype=np.float32)
    if arr.shape[:2] != shape:
        raise ValueError(f"{name} guide must match pixel height and width")
    if arr.ndim == 2:
        arr = arr[:, :, None]
    elif arr.ndim != 3:
        raise ValueError(f"{name} guide must be a 2D or 3D array")
    if arr.shape[2] != channels:
        raise ValueError(f"{name} guide must have {channels} channel(s)")
    return arr


def edge_aware_denoise(linear_pixels, radius=1, sigma_color=0.08, amount=1.0, *, normal=None, albedo=None,
                       depth=None, sigma_normal=0.35, sigma_albedo=0.20, sigma_depth=1.0, passes=1):
    """Denoise linear RGB pixels with the guided edge-aware filter.

    Returns `linear_pixels` itself when disabled (radius <= 0 or amount <= 0).
    Optional normal/albedo guides are HxWx3; depth is HxW or HxWx1.
    """
    if radius <= 0 or amount <= 0.0:
        return linear_pixels
    src = np.asarray(linear_pixels, dtype=np.float32)
    shape = src.shape[:2]
    n = _guide("normal", normal, shape, 3)
    a = _guide("albedo", albedo, shape, 3)
    d = _guide("depth", depth, shape, 1)
    return nat.denoise(src, normal=n, albedo=a, depth=None if d is None else d[:, :, 0], radius=int(radius),
                       sigma_color=sigma_color, amount=min(max(float(amount), 0.0), 1.0), sigma_normal=sigma_normal,
                       sigma_albedo=sigma_albedo, sigma_depth=sigma_depth, passes=int(passes))


def linear_to_display(linear_pixels):
    return np.sqrt(np.minimum(np.maximum(linear_pixels, 0.0), 1.0)).astype(np.float32)
