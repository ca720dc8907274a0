import numpy as np


class Image:
    """(height, width, 3) float32 display-space pixel buffer."""

    def __init__(self, width, height):
        self._width, self._height = width, height
        self._pixels = np.zeros((height, width, 3), dtype=np.float32)

    width = property(lambda s: s._width)
    height = property(lambda s: s._height)
    aspect_ratio = property(lambda s: s._width / s._height)
    pixels = property(lambda s: s._pixels)

    def read_pixel(self, x, y):
        return self._pixels[y, x]

    def clear(self):
        self._pixels[:] = 0

    def __repr__(self):
        return f"Image({self._width}x{self._height})"
