"""Analytic primitives rendered as object slots (sphere, plane, cube)."""
from core import Vec3


class Primitive:
    is_infinite = False


class Sphere(Primitive):
    def __init__(self, radius=1.0):
        self._radius = radius

    def taichi_type_id(self):
        return 0

    def __repr__(self):
        return f"Sphere(radius={self._radius})"


class Plane(Primitive):
    is_infinite = True

    def __init__(self, normal=Vec3(0, 1, 0), distance=0):
        self._normal = normal.normalize()
        self._distance = distance

    def taichi_type_id(self):
        return 1


class Cube(Primitive):
    def __init__(self, side_length=1.0):
        self._side_length = side_length

    def taichi_type_id(self):
        return 2
