"""Triangle meshes: Triangle / Mesh (object per triangle) and IndexedMesh
(shared position / normal / uv arrays with per-triangle index tables)."""
import numpy as np

from core import Vec2, Vec3


class Triangle:
    def __init__(self, v0, v1, v2, n0=None, n1=None, n2=None, uv0=None, uv1=None, uv2=None, group="default"):
        self._v0, self._v1, self._v2 = v0, v1, v2
        self._n0, self._n1, self._n2 = n0, n1, n2
        self._uv0, self._uv1, self._uv2 = uv0, uv1, uv2
        self._normal = (v1 - v0).cross(v2 - v0).normalize()
        self._group = group

    @property
    def group(self):
        return self._group

    def taichi_type_id(self):
        return 4


class Mesh:
    def __init__(self, triangles=None, name=""):
        from core.bvh import BVHNode
        self._triangles = triangles or []
        self._name = name
        # building the object BVH orders the triangle list (see core.bvh)
        self._bvh = BVHNode(self._triangles) if self._triangles else None

    is_infinite = False

    def taichi_type_id(self):
        return 5

    def __repr__(self):
        return f"Mesh(num_triangles={len(self._triangles)})"


class IndexedMesh:
    """Positions + index tables.  `build_bvh` is accepted for API compatibility;
    the GPU path builds its own BVH over all scene triangles."""

    is_infinite = False

    def __init__(self, positions, tri_pos_idx, normals=None, tri_normal_idx=None, uvs=None, tri_uv_idx=None,
                 groups=None, tri_group_idx=None, name="", build_bvh=True):
        self._positions = np.asarray(positions, dtype=np.float64).reshape((-1, 3))
        self._tri_pos_idx = np.asarray(tri_pos_idx, dtype=np.int32).reshape((-1, 3))
        n = len(self._tri_pos_idx)
        self._normals = None if normals is None else np.asarray(normals, dtype=np.float64).reshape((-1, 3))
        self._tri_normal_idx = self._table(tri_normal_idx, n)
        self._uvs = None if uvs is None else np.asarray(uvs, dtype=np.float64).reshape((-1, 2))
        self._tri_uv_idx = self._table(tri_uv_idx, n)
        self._groups = list(groups) if groups else ["default"]
        self._tri_group_idx = (np.zeros(n, np.int32) if tri_group_idx is None
                               else np.asarray(tri_group_idx, dtype=np.int32).reshape((-1,)))
        self._name = name

    @staticmethod
    def _table(v, n):
        if v is None:
            return np.full((n, 3), -1, dtype=np.int32)
        return np.asarray(v, dtype=np.int32).reshape((n, 3))

    vertex_count = property(lambda s: len(s._positions))
    triangle_count = property(lambda s: len(s._tri_pos_idx))
    groups = property(lambda s: list(s._groups))

    def triangle_vertices(self, tri_i):
        """Vec3 corners of triangle tri_i (scene/mesh.py:382-384)."""
        row = self._positions[self._tri_pos_idx[tri_i]]
        return tuple(Vec3(float(r[0]), float(r[1]), float(r[2])) for r in row)

    def group_for_triangle(self, tri_i):
        """Material group name of triangle tri_i (scene/mesh.py:394-395)."""
        return self._groups[int(self._tri_group_idx[tri_i])]

    def taichi_type_id(self):
        return 6

    @staticmethod
    def _normalize_rows(rows):
        length = np.linalg.norm(rows, axis=1)
        out = rows.copy()
        ok = length > 1e-12
        out[ok] /= length[ok, None]
        return out

    @staticmethod
    def _apply_point(m, pts):
        a = np.asarray(m.rows, dtype=np.float64)
        out = pts @ a[:3, :3].T + a[:3, 3]
        w = pts @ a[3, :3].T + a[3, 3]
        div = np.abs(w) > 1e-12
        out[div] /= w[div, None]
        return out

    @staticmethod
    def _apply_vector(m, v):
        a = np.asarray(m.rows, dtype=np.float64)
        return v @ a[:3, :3].T

    def indexed_triangle_arrays(self, matrix=None, normal_matrix=None, dtype=np.float32):
        """Per-triangle arrays in world space (scene/mesh.py:397-430 contract):
        v0..v2 / n0..n2 (T,3), uv0..uv2 (T,2), has_uv, group_idx, groups."""
        n = self.triangle_count
        tv = self._positions[self._tri_pos_idx].reshape((-1, 3))
        if matrix is not None:
            tv = self._apply_point(matrix, tv)
        tv = tv.reshape((n, 3, 3))
        raw = self._positions[self._tri_pos_idx]
        face = self._normalize_rows(np.cross(raw[:, 1] - raw[:, 0], raw[:, 2] - raw[:, 0]))
        tn = np.repeat(face[:, None, :], 3, axis=1)
        if self._normals is not None:
            ok = np.all(self._tri_normal_idx >= 0, axis=1)
            if np.any(ok):
                tn[ok] = self._normals[self._tri_normal_idx[ok]]
        tn = tn.reshape((-1, 3))
        if normal_matrix is not None:
            tn = self._apply_vector(normal_matrix, tn)
        tn = self._normalize_rows(tn).reshape((n, 3, 3))
        out = {
            "v0": tv[:, 0].astype(dtype), "v1": tv[:, 1].astype(dtype), "v2": tv[:, 2].astype(dtype),
            "n0": tn[:, 0].astype(dtype), "n1": tn[:, 1].astype(dtype), "n2": tn[:, 2].astype(dtype),
        }
        out.update(self.indexed_uv_arrays(dtype))
        out["group_idx"] = self._tri_group_idx.astype(np.int32)
        out["groups"] = list(self._groups)
        return out

    def indexed_uv_arrays(self, dtype=np.float32):
        """uv0..uv2 (T,2) and has_uv (T,) of indexed_triangle_arrays."""
        n = self.triangle_count
        tuv = np.zeros((n, 3, 2), np.float64)
        if self._uvs is not None:
            ok = np.all(self._tri_uv_idx >= 0, axis=1)
            if np.any(ok):
                tuv[ok] = self._uvs[self._tri_uv_idx[ok]]
        return {"uv0": tuv[:, 0].astype(dtype), "uv1": tuv[:, 1].astype(dtype), "uv2": tuv[:, 2].astype(dtype),
                "has_uv": np.all(self._tri_uv_idx >= 0, axis=1).astype(np.int32)}

    def __repr__(self):
        return f"IndexedMesh(vertices={self.vertex_count}, triangles={self.triangle_count}, groups={len(self._groups)})"


def indexed_triangle_arrays(mesh, matrix=None, normal_matrix=None, dtype=np.float32):
    if not isinstance(mesh, IndexedMesh):
        raise TypeError("indexed_triangle_arrays expects an IndexedMesh")
    return mesh.indexed_triangle_arrays(matrix, normal_matrix, dtype=dtype)


__all__ = ["Triangle", "Mesh", "IndexedMesh", "indexed_triangle_arrays", "Vec2", "Vec3"]
