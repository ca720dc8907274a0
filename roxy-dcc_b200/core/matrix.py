"""Row-major 4x4 matrices for scene transforms.

The composition convention is the reference's (core/matrix.py): column
vectors, world = T * (Tp) * R * Sh * S * (Tp^-1), R built from per-axis
rotations in degrees in the given Euler order, and the no-shear inverse as
S^-1 * R^T * T^-1.  Products sum left to right so the world-space triangles
handed to the GPU round the same way.
"""
import math

from core.enums import RotationOrder


class Mat4x4:
    __slots__ = ("rows",)

    def __init__(self, rows=None):
        self.rows = rows if rows is not None else [[0.0] * 4 for _ in range(4)]

    @classmethod
    def identity(cls):
        return cls([[1 if i == j else 0 for j in range(4)] for i in range(4)])

    @classmethod
    def translation(cls, x, y, z):
        return cls([[1, 0, 0, x], [0, 1, 0, y], [0, 0, 1, z], [0, 0, 0, 1]])

    @classmethod
    def scale(cls, x, y, z):
        return cls([[x, 0, 0, 0], [0, y, 0, 0], [0, 0, z, 0], [0, 0, 0, 1]])

    @classmethod
    def shear(cls, a, b, c):
        return cls([[1, a, b, 0], [0, 1, c, 0], [0, 0, 1, 0], [0, 0, 0, 1]])

    @classmethod
    def rotation_x(cls, deg):
        c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
        return cls([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]])

    @classmethod
    def rotation_y(cls, deg):
        c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
        return cls([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1]])

    @classmethod
    def rotation_z(cls, deg):
        c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
        return cls([[c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])

    @classmethod
    def rotation(cls, rot, order=RotationOrder.XYZ):
        m = {"x": cls.rotation_x(rot.x), "y": cls.rotation_y(rot.y), "z": cls.rotation_z(rot.z)}
        seq = RotationOrder(order).value
        return m[seq[0]] * m[seq[1]] * m[seq[2]]

    @classmethod
    def from_trs(cls, translation, rotation, scale, shear=None, pivot=None, rotation_order=RotationOrder.XYZ):
        T = cls.translation(translation.x, translation.y, translation.z)
        R = cls.rotation(rotation, rotation_order)
        S = cls.scale(scale.x, scale.y, scale.z)
        Sh = cls.shear(shear.x, shear.y, shear.z) if shear else cls.identity()
        if pivot:
            P = cls.translation(pivot.x, pivot.y, pivot.z)
            Pi = cls.translation(-pivot.x, -pivot.y, -pivot.z)
            return T * P * R * Sh * S * Pi
        return T * R * Sh * S

    @classmethod
    def inverse_trs(cls, translation, rotation, scale, shear=None, pivot=None, rotation_order=RotationOrder.XYZ):
        has_shear = shear and (shear.x or shear.y or shear.z)
        has_pivot = pivot and (pivot.x or pivot.y or pivot.z)
        if has_shear or has_pivot:
            return cls.from_trs(translation, rotation, scale, shear, pivot, rotation_order).inverse()
        S_inv = cls.scale(1 / scale.x, 1 / scale.y, 1 / scale.z)
        R_t = cls.rotation(rotation, rotation_order).transpose()
        T_inv = cls.translation(-translation.x, -translation.y, -translation.z)
        return S_inv * R_t * T_inv

    def __mul__(self, o):
        if isinstance(o, Mat4x4):
            a, b = self.rows, o.rows
            return Mat4x4([[sum(a[i][k] * b[k][j] for k in range(4)) for j in range(4)] for i in range(4)])
        return Mat4x4([[v * o for v in r] for r in self.rows])

    def transpose(self):
        return Mat4x4([[self.rows[j][i] for j in range(4)] for i in range(4)])

    def inverse(self):
        """Gauss-Jordan elimination with partial pivoting."""
        aug = [list(self.rows[i]) + [1 if i == j else 0 for j in range(4)] for i in range(4)]
        for col in range(4):
            piv = max(range(col, 4), key=lambda r: abs(aug[r][col]))
            aug[col], aug[piv] = aug[piv], aug[col]
            if abs(aug[col][col]) < 1e-10:
                raise ValueError("Matrix is not invertible")
            s = aug[col][col]
            aug[col] = [v / s for v in aug[col]]
            for r in range(4):
                if r != col:
                    f = aug[r][col]
                    aug[r] = [aug[r][k] - f * aug[col][k] for k in range(8)]
        return Mat4x4([row[4:] for row in aug])

    def transform_point(self, p):
        from core.vectors import Vec3
        px, py, pz = p
        r = self.rows
        x = px * r[0][0] + py * r[0][1] + pz * r[0][2] + r[0][3]
        y = px * r[1][0] + py * r[1][1] + pz * r[1][2] + r[1][3]
        z = px * r[2][0] + py * r[2][1] + pz * r[2][2] + r[2][3]
        w = px * r[3][0] + py * r[3][1] + pz * r[3][2] + r[3][3]
        if w != 0:
            return Vec3(x / w, y / w, z / w)
        return Vec3(x, y, z)

    def transform_vector(self, v):
        from core.vectors import Vec3
        vx, vy, vz = v
        r = self.rows
        return Vec3(vx * r[0][0] + vy * r[0][1] + vz * r[0][2], vx * r[1][0] + vy * r[1][1] + vz * r[1][2],
                    vx * r[2][0] + vy * r[2][1] + vz * r[2][2])

    def __eq__(self, o):
        return isinstance(o, Mat4x4) and all(abs(self.rows[i][j] - o.rows[i][j]) < 1e-9
                                             for i in range(4) for j in range(4))

    def __repr__(self):
        return f"Mat4x4({self.rows})"
