"""TRS transform with cached world / inverse matrices."""
from core.enums import RotationOrder
from core.matrix import Mat4x4
from core.vectors import Vec3


class Transform:
    def __init__(self, translation=None, rotation=None, scale=None, shear=None, pivot=None, matrix=None,
                 inverse_matrix=None, rotation_order=RotationOrder.XYZ, shape=None):
        self._translation = translation if translation is not None else Vec3(0, 0, 0)
        self._rotation = rotation if rotation is not None else Vec3(0, 0, 0)
        self._scale = scale if scale is not None else Vec3(1, 1, 1)
        self._shear = shear if shear is not None else Vec3(0, 0, 0)
        self._pivot = pivot if pivot is not None else Vec3(0, 0, 0)
        self._rotation_order = rotation_order
        self._matrix_mode = matrix is not None
        if self._matrix_mode:
            rows = matrix.rows if isinstance(matrix, Mat4x4) else matrix
            self._matrix = Mat4x4([[float(v) for v in r] for r in rows])
            if inverse_matrix is not None:
                irows = inverse_matrix.rows if isinstance(inverse_matrix, Mat4x4) else inverse_matrix
                self._inverse = Mat4x4([[float(v) for v in r] for r in irows])
            else:
                self._inverse = self._matrix.inverse()
        else:
            self._rebuild()

    def _rebuild(self):
        args = (self._translation, self._rotation, self._scale, self._shear, self._pivot, self._rotation_order)
        self._matrix = Mat4x4.from_trs(*args)
        self._inverse = Mat4x4.inverse_trs(*args)

    def _set(self, name, value):
        setattr(self, name, value)
        self._matrix_mode = False
        self._rebuild()

    translation = property(lambda s: s._translation, lambda s, v: s._set("_translation", v))
    rotation = property(lambda s: s._rotation, lambda s, v: s._set("_rotation", v))
    scale = property(lambda s: s._scale, lambda s, v: s._set("_scale", v))
    shear = property(lambda s: s._shear, lambda s, v: s._set("_shear", v))
    pivot = property(lambda s: s._pivot, lambda s, v: s._set("_pivot", v))
    rotation_order = property(lambda s: s._rotation_order, lambda s, v: s._set("_rotation_order", v))

    @property
    def matrix_mode(self):
        return self._matrix_mode

    @property
    def world_matrix(self):
        return self._matrix

    @property
    def world_inverse_matrix(self):
        return self._inverse

    @property
    def matrix(self):
        return self._matrix

    @matrix.setter
    def matrix(self, m):
        self._matrix_mode = True
        self._matrix = m if isinstance(m, Mat4x4) else Mat4x4(m)
        self._inverse = self._matrix.inverse()
