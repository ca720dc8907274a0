"""ImageTexture with the reference's interface (scene/textures.py:6-110):
an RGB image sampled with repeating uvs and bilinear filtering.  The GPU
path uploads `load_pixels_u8()` and samples it in the shading kernel."""
import numpy as np

from core import Color


class ImageTexture:
    def __init__(self, path=None, pixels=None, flip_v=True):
        if path is None and pixels is None:
            raise ValueError("ImageTexture needs either a path or pixel array")
        self.path = str(path) if path is not None else None
        self._pixels = None if pixels is None else self._coerce_pixels(pixels)
        self.flip_v = flip_v

    @classmethod
    def from_array(cls, pixels, flip_v=True):
        return cls(pixels=pixels, flip_v=flip_v)

    @staticmethod
    def _coerce_pixels(pixels):
        arr = np.asarray(pixels, dtype=np.float32)
        if arr.ndim != 3 or arr.shape[2] < 3:
            raise ValueError("texture pixels must be an HxWx3 array")
        arr = arr[:, :, :3]
        if arr.size and arr.max() > 1.0:
            arr = arr / 255.0
        return np.clip(arr, 0.0, 1.0)

    def _load_pixels(self):
        if self._pixels is not None:
            return self._pixels
        # image files are decoded by pygame in the reference; it is not part
        # of this package
        raise RuntimeError("pygame is required to load image textures")

    def load_pixels_u8(self, max_size=None):
        """HxWx3 uint8 pixels, as the GPU path uploads them."""
        if self.path is None:
            pixels = self._load_pixels()
            return np.clip(pixels * 255.0 + 0.5, 0, 255).astype(np.uint8)
        raise RuntimeError("pygame is required to load image textures")

    def sample(self, uv):
        pixels = self._load_pixels()
        h, w = pixels.shape[:2]
        if h == 0 or w == 0:
            return Color(1, 1, 1)
        u = float(uv[0]) % 1.0
        v = float(uv[1]) % 1.0
        if self.flip_v:
            v = 1.0 - v
        x = u * (w - 1)
        y = v * (h - 1)
        x0, y0 = int(np.floor(x)), int(np.floor(y))
        x1, y1 = min(x0 + 1, w - 1), min(y0 + 1, h - 1)
        tx, ty = x - x0, y - y0
        c0 = pixels[y0, x0] * (1.0 - tx) + pixels[y0, x1] * tx
        c1 = pixels[y1, x0] * (1.0 - tx) + pixels[y1, x1] * tx
        c = c0 * (1.0 - ty) + c1 * ty
        return Color(float(c[0]), float(c[1]), float(c[2]))

    def to_dict(self):
        if self.path is None:
            return None
        return {"type": "image", "path": self.path, "flip_v": self.flip_v}


def create_texture_from_dict(data):
    if data is None:
        return None
    if data.get("type") == "image":
        return ImageTexture(data["path"], flip_v=data.get("flip_v", True))
    raise ValueError(f"Unknown texture type: {data.get('type')}")
