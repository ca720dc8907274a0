"""Scene graph node: shapes, a TRS transform and children."""
import math

from core import Color, RotationOrder, Transform, Vec3


def _point(r, px, py, pz):
    """Mat4x4.transform_point on rows `r`: the same operations, as a list."""
    x = px * r[0][0] + py * r[0][1] + pz * r[0][2] + r[0][3]
    y = px * r[1][0] + py * r[1][1] + pz * r[1][2] + r[1][3]
    z = px * r[2][0] + py * r[2][1] + pz * r[2][2] + r[2][3]
    w = px * r[3][0] + py * r[3][1] + pz * r[3][2] + r[3][3]
    return [x / w, y / w, z / w] if w != 0 else [x, y, z]


def _vec_len(r, vx, vy, vz):
    """Mat4x4.transform_vector(...).length() on rows `r`, the same operations."""
    x = vx * r[0][0] + vy * r[0][1] + vz * r[0][2]
    y = vx * r[1][0] + vy * r[1][1] + vz * r[1][2]
    z = vx * r[2][0] + vy * r[2][1] + vz * r[2][2]
    return math.sqrt(x * x + y * y + z * z)


class SceneObject:
    def __init__(self, shapes=None, name="", translation=None, rotation=None, scale=None, shear=None, pivot=None,
                 matrix=None, inverse_matrix=None, visible=True, renderable=True, selectable=True,
                 rotation_order=RotationOrder.XYZ, shape=None, material=None):
        self._name = name
        self._shapes = list(shapes) if shapes else []
        self._children = []
        self._parent = None
        self._visible = visible
        self._renderable = renderable
        self._selectable = selectable
        if shape is not None:
            from scene.shape import Shape
            self._shapes.append(Shape(shape, {"default": material} if material is not None else {}, name=name))
        self._transform = Transform(translation=translation, rotation=rotation, scale=scale, shear=shear,
                                    pivot=pivot, matrix=matrix, inverse_matrix=inverse_matrix,
                                    rotation_order=rotation_order)

    # hierarchy
    def add_child(self, child):
        child._parent = self
        if child not in self._children:
            self._children.append(child)
        return child

    def remove_child(self, child):
        child._parent = None
        if child in self._children:
            self._children.remove(child)

    children = property(lambda s: list(s._children))
    parent = property(lambda s: s._parent)
    name = property(lambda s: s._name)
    shapes = property(lambda s: s._shapes)
    transform = property(lambda s: s._transform)

    @property
    def world_matrix(self):
        if self._parent:
            return self._parent.world_matrix * self._transform.world_matrix
        return self._transform.world_matrix

    @property
    def world_inverse_matrix(self):
        if self._parent:
            return self._transform.world_inverse_matrix * self._parent.world_inverse_matrix
        return self._transform.world_inverse_matrix

    @property
    def world_inverse_transpose_matrix(self):
        return self.world_inverse_matrix.transpose()

    @property
    def shape(self):
        return self._shapes[0].geometry if self._shapes else None

    @property
    def material(self):
        return self._shapes[0].material_for_group("default") if self._shapes else None

    @material.setter
    def material(self, value):
        if self._shapes:
            self._shapes[0]._material_groups["default"] = value

    @property
    def renderable(self):
        return self._renderable

    @renderable.setter
    def renderable(self, v):
        self._renderable = v

    @property
    def visible(self):
        return self._visible

    @visible.setter
    def visible(self, v):
        self._visible = v

    @staticmethod
    def material_record(mat):
        """GPU material record of the reference (scene_object.py taichi_export)."""
        mt = mat.taichi_type_id()
        params = mat.taichi_params()
        return {"albedo": list(mat._albedo), "mat_type": mt,
                "roughness": params[0] if mt in (1, 4) else 0.0,
                "ior": params[0] if mt == 2 else 1.0,
                "emission": params[0] if mt == 3 else 0.0}

    def taichi_export(self):
        """World-space object slot(s) in the reference's flat layout: spheres
        keep max-axis-scaled radii, cubes keep axis-aligned half extents
        (rotation ignored), planes carry a world normal and offset, triangles
        carry world vertices."""
        from scene.materials import Diffuse
        from scene.mesh import Mesh, Triangle
        from scene.primitives import Cube, Plane, Sphere
        shape = self.shape
        if shape is None:
            return []
        M = self.world_matrix
        mat = self.material or Diffuse(Color(0.8, 0.8, 0.8))
        rec = self.material_record(mat)
        zero = [0.0, 0.0, 0.0]
        if isinstance(shape, Sphere):
            # M.transform_point(Vec3(0, 0, 0)) and the lengths of M applied to
            # the unit axes, in the same arithmetic without the Vec3 objects
            r = M.rows
            c = _point(r, 0, 0, 0)
            s = max(_vec_len(r, 1, 0, 0), _vec_len(r, 0, 1, 0), _vec_len(r, 0, 0, 1))
            return {"type": 0, "center": c, "radius": shape._radius * s, "normal": [0.0, 1.0, 0.0], "offset": 0.0,
                    "extra": zero, **rec}
        if isinstance(shape, Plane):
            inv = self.world_inverse_matrix
            n = inv.transpose().transform_vector(shape._normal).normalize()
            d = shape._distance
            p = M.transform_point(Vec3(shape._normal.x * -d, shape._normal.y * -d, shape._normal.z * -d))
            return {"type": 1, "center": zero, "radius": 0.0, "normal": list(n), "offset": -n.dot(p),
                    "extra": zero, **rec}
        if isinstance(shape, Cube):
            c = list(M.transform_point(Vec3(0, 0, 0)))
            h = shape._side_length / 2
            sx = M.transform_vector(Vec3(1, 0, 0)).length()
            sy = M.transform_vector(Vec3(0, 1, 0)).length()
            sz = M.transform_vector(Vec3(0, 0, 1)).length()
            return {"type": 2, "center": c, "radius": 0.0, "normal": [0.0, 1.0, 0.0], "offset": 0.0,
                    "extra": [h * sx, h * sy, h * sz], **rec}

        def tri_slot(tri):
            m = self._shapes[0].material_for_group(getattr(tri, "group", "default")) or mat
            return {"type": 4, "center": zero, "radius": 0.0, "normal": [0.0, 1.0, 0.0], "offset": 0.0,
                    "extra": zero, "v0": list(M.transform_point(tri._v0)), "v1": list(M.transform_point(tri._v1)),
                    "v2": list(M.transform_point(tri._v2)), **self.material_record(m)}

        if isinstance(shape, Triangle):
            return tri_slot(shape)
        if isinstance(shape, Mesh):
            return [tri_slot(t) for t in shape._triangles]
        raise NotImplementedError(f"taichi_export not supported for {type(shape).__name__}")

    def __repr__(self):
        return f"SceneObject(name={self._name!r}, shapes={len(self._shapes)}, children={len(self._children)})"
