import math

from core import Point3, Vec3


class Camera:
    """Pinhole camera: position, orthonormal forward / right / up, vertical FOV (degrees)."""

    def __init__(self, position=Point3(), forward=Vec3(0, 0, -1), up=Vec3(0, 1, 0), fov=90, width=800,
                 height=600, name="camera"):
        self._position = position
        self._forward = forward.normalize()
        self._right = self._forward.cross(up.normalize()).normalize()
        self._up = self._right.cross(self._forward).normalize()
        self._fov = fov
        self._aspect_ratio = width / height if height != 0 else 1.0
        self.name = name

    position = property(lambda s: s._position)
    forward = property(lambda s: s._forward)
    up = property(lambda s: s._up)
    right = property(lambda s: s._right)
    fov = property(lambda s: s._fov)
    aspect_ratio = property(lambda s: s._aspect_ratio)

    @position.setter
    def position(self, p):
        self._position = p

    def set_width_height(self, width, height):
        self._aspect_ratio = width / height if height != 0 else 1.0

    @property
    def fov_tan(self):
        return math.tan(math.radians(self._fov) / 2)

    def __repr__(self):
        return f"Camera(position={self._position}, forward={self._forward}, fov={self._fov})"
