"""Sampling helpers (rendering/sampling.py API).

The GPU path draws every random number from a counter-based Philox4x32-10
generator keyed by (pixel, sample, bounce, slot) and jitters camera rays by
fract(per-pixel phase + (frame + 1) * R2); `philox4x32` and
`gpu_pixel_sample_offset` restate those in Python.  `pixel_sample_offset`
keeps the reference's sin-hash form for host callers.
"""
import math

_R2_X = 0.7548776662466927
_R2_Y = 0.5698402909980532
_M0, _M1 = 0xD2511F53, 0xCD9E8D57
_W0, _W1 = 0x9E3779B9, 0xBB67AE85
_KEY_HI = 0x5EEDC0DE


def _fract(v):
    return v - math.floor(v)


def _hash_float(x, y, salt=0):
    return _fract(math.sin(x * 127.1 + y * 311.7 + salt * 74.7) * 43758.5453123)


def pixel_sample_offset(x, y, frame):
    """Low-discrepancy pixel offset in [0, 1) with a per-pixel phase shift."""
    i = frame + 1
    return (_fract(_hash_float(x, y, 0) + i * _R2_X), _fract(_hash_float(x, y, 1) + i * _R2_Y))


def philox4x32(counter, key):
    """Philox4x32-10 (Salmon et al., SC'11) on a 4-word counter, 2-word key."""
    c0, c1, c2, c3 = (int(v) & 0xFFFFFFFF for v in counter)
    k0, k1 = (int(v) & 0xFFFFFFFF for v in key)
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF, \
                         ((p0 >> 32) ^ c3 ^ k1) & 0xFFFFFFFF, p0 & 0xFFFFFFFF
        k0 = (k0 + _W0) & 0xFFFFFFFF
        k1 = (k1 + _W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def uniform01(word):
    return (word >> 8) * (1.0 / 16777216.0)


def gpu_pixel_sample_offset(x, y, frame, width, seed=0):
    """Camera jitter the GPU path uses for pixel (x, y) at `frame` (float64 view)."""
    ph = philox4x32(((y * width + x), 0xFFFFFFFF, 0xFFFFFFFF, 0), (seed, _KEY_HI))
    i = frame + 1
    return _fract(uniform01(ph[0]) + i * _R2_X), _fract(uniform01(ph[1]) + i * _R2_Y)


def clamp_color_sample(color, sample_clamp):
    if sample_clamp is None or sample_clamp <= 0:
        return color
    return color.__class__(min(max(color[0], 0.0), sample_clamp), min(max(color[1], 0.0), sample_clamp),
                           min(max(color[2], 0.0), sample_clamp))


def mis_power_weight(sample_pdf, other_pdf, beta=2.0):
    """Power-heuristic MIS weight of one sampled strategy."""
    a = max(0.0, sample_pdf) ** beta
    b = max(0.0, other_pdf) ** beta
    total = a + b
    return 0.0 if total <= 0.0 else a / total
