from enum import Enum


class RotationOrder(Enum):
    """Euler order of a Transform's rotation (degrees)."""

    XYZ = "xyz"
    ZYX = "zyx"
    XZY = "xzy"
    YXZ = "yxz"
    YZX = "yzx"
    ZXY = "zxy"
