"""Vec2 / Vec3 / Color / Point3 / Ray — the value types the scene API takes.

Same constructor and accessor surface as the reference's core/vectors.py
(immutable, iterable, indexable) so scenes written for it build unchanged.
"""
import math


class Vec2:
    __slots__ = ("_x", "_y")

    def __init__(self, x=0.0, y=0.0):
        self._x, self._y = x, y

    x = property(lambda s: s._x)
    y = property(lambda s: s._y)

    def __add__(self, o):
        return self.__class__(self._x + o._x, self._y + o._y)

    def __sub__(self, o):
        return self.__class__(self._x - o._x, self._y - o._y)

    def __mul__(self, s):
        return self.__class__(self._x * s, self._y * s)

    __rmul__ = __mul__

    def __iter__(self):
        yield self._x
        yield self._y

    def __getitem__(self, i):
        return (self._x, self._y)[i]

    def __eq__(self, o):
        return isinstance(o, Vec2) and self._x == o._x and self._y == o._y

    def __hash__(self):
        return hash((self._x, self._y))

    def __repr__(self):
        return f"Vec2({self._x}, {self._y})"

    def to_dict(self):
        return [self._x, self._y]

    @classmethod
    def from_dict(cls, d):
        return cls(d[0], d[1])


class Vec3:
    __slots__ = ("_x", "_y", "_z")

    def __init__(self, x=0.0, y=0.0, z=0.0):
        self._x, self._y, self._z = x, y, z

    x = property(lambda s: s._x)
    y = property(lambda s: s._y)
    z = property(lambda s: s._z)

    def __add__(self, o):
        return self.__class__(self._x + o._x, self._y + o._y, self._z + o._z)

    def __sub__(self, o):
        return self.__class__(self._x - o._x, self._y - o._y, self._z - o._z)

    def __mul__(self, o):
        if isinstance(o, Vec3):
            return self.__class__(self._x * o._x, self._y * o._y, self._z * o._z)
        return self.__class__(self._x * o, self._y * o, self._z * o)

    __rmul__ = __mul__

    def __truediv__(self, s):
        return self * (1.0 / s)

    def __neg__(self):
        return self.__class__(-self._x, -self._y, -self._z)

    def dot(self, o):
        return self._x * o._x + self._y * o._y + self._z * o._z

    def cross(self, o):
        return self.__class__(self._y * o._z - self._z * o._y, self._z * o._x - self._x * o._z,
                              self._x * o._y - self._y * o._x)

    def length_sq(self):
        return self.dot(self)

    def length(self):
        return math.sqrt(self.length_sq())

    def normalize(self):
        m = self.length()
        return self / m if m > 0 else self.__class__(0.0, 0.0, 0.0)

    def __iter__(self):
        yield self._x
        yield self._y
        yield self._z

    def __getitem__(self, i):
        return (self._x, self._y, self._z)[i]

    def __len__(self):
        return 3

    def __eq__(self, o):
        return isinstance(o, Vec3) and (self._x, self._y, self._z) == (o._x, o._y, o._z)

    def __hash__(self):
        return hash((self._x, self._y, self._z))

    def __repr__(self):
        return f"{self.__class__.__name__}({self._x}, {self._y}, {self._z})"

    def to_dict(self):
        return [self._x, self._y, self._z]

    @classmethod
    def from_dict(cls, d):
        return cls(d[0], d[1], d[2])


class Color(Vec3):
    __slots__ = ()
    r = property(lambda s: s._x)
    g = property(lambda s: s._y)
    b = property(lambda s: s._z)


Point3 = Vec3


class Ray:
    __slots__ = ("_origin", "_direction")

    def __init__(self, origin, direction):
        self._origin, self._direction = origin, direction.normalize()

    origin = property(lambda s: s._origin)
    direction = property(lambda s: s._direction)

    def at(self, t):
        return self._origin + self._direction * t
