"""Value types and transforms consumed by the scene API."""
from core.enums import RotationOrder
from core.matrix import Mat4x4
from core.transform import Transform
from core.vectors import Color, Point3, Ray, Vec2, Vec3

__all__ = ["Vec2", "Vec3", "Color", "Ray", "Point3", "Mat4x4", "RotationOrder", "Transform"]
