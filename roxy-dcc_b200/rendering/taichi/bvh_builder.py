"""TriangleBatch and GPUBVHBuilder with the reference's call signatures
(rendering/taichi/bvh_builder.py:8-655), building on the device.

`GPUBVHBuilder.build` gathers and validates triangles on the host, dedupes
materials into a palette (same keys and first-seen order as the reference),
and hands the triangles to libroxy_cuda.so:

* method "morton" (default, the reference's): Morton codes, stable radix sort
  and the count-median tree are computed on the GPU; `nodes`,
  `ordered_tris` and the `_ordered_*` arrays equal the reference builder's
  output bit for bit.
* method "lbvh": Karras LBVH with SAH leaf collapse (the renderer's tree;
  `nodes` then only reports its length).
* method "median": the reference's longest-axis median split, a host-side
  legacy path kept for API compatibility; the tree is uploaded as given.
"""
from dataclasses import dataclass

import numpy as np

import roxy_native as nat


@dataclass
class TriangleBatch:
    v0: np.ndarray
    v1: np.ndarray
    v2: np.ndarray
    n0: np.ndarray
    n1: np.ndarray
    n2: np.ndarray
    mat_type: np.ndarray
    albedo: np.ndarray
    roughness: np.ndarray
    ior: np.ndarray
    emission: np.ndarray
    uv0: np.ndarray = None
    uv1: np.ndarray = None
    uv2: np.ndarray = None
    has_uv: np.ndarray = None
    texture_idx: np.ndarray = None
    mat_idx: np.ndarray = None
    mat_palette: list = None

    def __post_init__(self):
        v3 = lambda a: np.asarray(a, dtype=np.float32).reshape((-1, 3))  # noqa: E731
        self.v0, self.v1, self.v2 = v3(self.v0), v3(self.v1), v3(self.v2)
        self.n0, self.n1, self.n2 = v3(self.n0), v3(self.n1), v3(self.n2)
        n = len(self.v0)
        self.mat_type = np.asarray(self.mat_type, dtype=np.int32).reshape((-1,))
        self.albedo = v3(self.albedo)
        self.roughness = np.asarray(self.roughness, dtype=np.float32).reshape((-1,))
        self.ior = np.asarray(self.ior, dtype=np.float32).reshape((-1,))
        self.emission = np.asarray(self.emission, dtype=np.float32).reshape((-1,))
        v2_ = lambda a: (np.zeros((n, 2), np.float32) if a is None  # noqa: E731
                         else np.asarray(a, dtype=np.float32).reshape((-1, 2)))
        self.uv0, self.uv1, self.uv2 = v2_(self.uv0), v2_(self.uv1), v2_(self.uv2)
        self.has_uv = (np.zeros(n, np.int32) if self.has_uv is None
                       else np.asarray(self.has_uv, dtype=np.int32).reshape((-1,)))
        n_mat_rows = n if self.mat_idx is None else len(self.mat_type)
        self.texture_idx = (np.full(n_mat_rows, -1, np.int32) if self.texture_idx is None
                            else np.asarray(self.texture_idx, dtype=np.int32).reshape((-1,)))
        geo = {len(a) for a in (self.v0, self.v1, self.v2, self.n0, self.n1, self.n2, self.uv0, self.uv1,
                                self.uv2, self.has_uv)}
        if len(geo) != 1:
            raise ValueError("TriangleBatch geometry arrays must all have the same length")
        mats = {len(a) for a in (self.mat_type, self.albedo, self.roughness, self.ior, self.emission,
                                 self.texture_idx)}
        if self.mat_idx is None:
            if len(mats) != 1 or next(iter(mats)) != n:
                raise ValueError("TriangleBatch per-triangle material arrays must match triangle count")
        else:
            self.mat_idx = np.asarray(self.mat_idx, dtype=np.int32).reshape((-1,))
            if len(self.mat_idx) != n:
                raise ValueError("TriangleBatch mat_idx must match triangle count")
            if len(mats) != 1:
                raise ValueError("TriangleBatch material palette arrays must all have the same length")
            if self.mat_palette is None:
                self.mat_palette = [self._record(i) for i in range(len(self.mat_type))]

    def _record(self, i):
        return {"type": int(self.mat_type[i]), "albedo": self.albedo[i].tolist(),
                "roughness": float(self.roughness[i]), "ior": float(self.ior[i]),
                "emission": float(self.emission[i]), "texture_idx": int(self.texture_idx[i])}

    @property
    def triangle_count(self):
        return len(self.v0)

    @classmethod
    def empty(cls):
        z3 = np.zeros((0, 3), np.float32)
        z = np.zeros(0, np.float32)
        zi = np.zeros(0, np.int32)
        return cls(z3, z3, z3, z3, z3, z3, zi, z3, z, z, z, uv0=np.zeros((0, 2), np.float32),
                   uv1=np.zeros((0, 2), np.float32), uv2=np.zeros((0, 2), np.float32), has_uv=zi, texture_idx=zi,
                   mat_idx=zi, mat_palette=[])

    @classmethod
    def from_dicts(cls, tris):
        if not tris:
            return cls.empty()
        col = lambda k, d=None: [t.get(k, d) if d is not None else t[k] for t in tris]  # noqa: E731
        return cls(col("v0"), col("v1"), col("v2"), col("n0"), col("n1"), col("n2"), col("mat_type"),
                   col("albedo"), col("roughness"), col("ior"), col("emission"), uv0=col("uv0", [0.0, 0.0]),
                   uv1=col("uv1", [0.0, 0.0]), uv2=col("uv2", [0.0, 0.0]), has_uv=col("has_uv", 0),
                   texture_idx=col("texture_idx", -1))

    @staticmethod
    def palette_record(m):
        """Palette entry of a material record, its values rounded to float32
        as the palette arrays store them."""
        return {"type": int(m["mat_type"]), "albedo": np.asarray(m["albedo"], np.float32).tolist(),
                "roughness": float(np.float32(m["roughness"])), "ior": float(np.float32(m["ior"])),
                "emission": float(np.float32(m["emission"])), "texture_idx": int(m.get("texture_idx", -1))}

    @classmethod
    def from_indexed_arrays(cls, arrays, material_by_group_idx):
        gidx = np.asarray(arrays["group_idx"], dtype=np.int32)
        used = np.unique(gidx)
        if len(used):
            remap = np.zeros(int(used.max()) + 1, np.int32)
            remap[used] = np.arange(len(used), dtype=np.int32)
            local = remap[gidx]
        else:
            local = gidx
        palette = [cls.palette_record(material_by_group_idx[int(g)]) for g in used]
        k = len(palette)
        return cls(arrays["v0"], arrays["v1"], arrays["v2"], arrays["n0"], arrays["n1"], arrays["n2"],
                   np.array([p["type"] for p in palette], np.int32).reshape(k),
                   np.array([p["albedo"] for p in palette], np.float32).reshape((k, 3)),
                   np.array([p["roughness"] for p in palette], np.float32).reshape(k),
                   np.array([p["ior"] for p in palette], np.float32).reshape(k),
                   np.array([p["emission"] for p in palette], np.float32).reshape(k),
                   uv0=arrays.get("uv0"), uv1=arrays.get("uv1"), uv2=arrays.get("uv2"), has_uv=arrays.get("has_uv"),
                   texture_idx=np.array([p["texture_idx"] for p in palette], np.int32).reshape(k),
                   mat_idx=local, mat_palette=palette)

    def as_palette_batch(self):
        """Same triangles with per-triangle materials turned into a palette."""
        if self.mat_idx is not None:
            return self
        n = self.triangle_count
        return TriangleBatch(self.v0, self.v1, self.v2, self.n0, self.n1, self.n2, self.mat_type, self.albedo,
                             self.roughness, self.ior, self.emission, uv0=self.uv0, uv1=self.uv1, uv2=self.uv2,
                             has_uv=self.has_uv, texture_idx=self.texture_idx,
                             mat_idx=np.arange(n, dtype=np.int32))

    @classmethod
    def concat(cls, batches):
        batches = [b for b in batches if b.triangle_count]
        if not batches:
            return cls.empty()
        if len(batches) == 1:
            return batches[0]
        cat = lambda name: np.concatenate([getattr(b, name) for b in batches])  # noqa: E731
        geo = dict(uv0=cat("uv0"), uv1=cat("uv1"), uv2=cat("uv2"), has_uv=cat("has_uv"))
        if all(b.mat_idx is None for b in batches):
            return cls(cat("v0"), cat("v1"), cat("v2"), cat("n0"), cat("n1"), cat("n2"), cat("mat_type"),
                       cat("albedo"), cat("roughness"), cat("ior"), cat("emission"), texture_idx=cat("texture_idx"),
                       **geo)
        # palette batches (mixed inputs are converted first; the reference
        # cannot concatenate a per-triangle batch with a palette batch)
        pb = [b.as_palette_batch() for b in batches]
        palette, idx = [], []
        for b in pb:
            idx.append(b.mat_idx + len(palette))
            palette.extend(b.mat_palette if b.mat_palette is not None else
                           [b._record(i) for i in range(len(b.mat_type))])
        k = len(palette)
        return cls(cat("v0"), cat("v1"), cat("v2"), cat("n0"), cat("n1"), cat("n2"),
                   np.array([m["type"] for m in palette], np.int32).reshape(k),
                   np.array([m["albedo"] for m in palette], np.float32).reshape((k, 3)),
                   np.array([m["roughness"] for m in palette], np.float32).reshape(k),
                   np.array([m["ior"] for m in palette], np.float32).reshape(k),
                   np.array([m["emission"] for m in palette], np.float32).reshape(k),
                   texture_idx=np.array([m.get("texture_idx", -1) for m in palette], np.int32).reshape(k),
                   mat_idx=np.concatenate(idx), mat_palette=palette, **geo)


class _NodeView:
    """List-like view of the reference-format node arrays (`builder.nodes`)."""

    def __init__(self, arrays=None, length=0):
        self._a = arrays
        self._n = len(arrays["left"]) if arrays is not None else length

    def __len__(self):
        return self._n

    def __getitem__(self, i):
        if self._a is None:
            raise IndexError("this BVH layout exposes no reference-format nodes")
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(self._n))]
        if i < 0:
            i += self._n
        if not 0 <= i < self._n:
            raise IndexError(i)
        a = self._a
        return {"aabb_min": a["node_min"][i].tolist(), "aabb_max": a["node_max"][i].tolist(),
                "left": int(a["left"][i]), "right": int(a["right"][i]), "tri_start": int(a["start"][i]),
                "tri_count": int(a["count"][i])}

    def __iter__(self):
        for i in range(self._n):
            yield self[i]


class GPUBVHBuilder:
    MAX_LEAF_SIZE = 8
    MAX_DEPTH = 32
    BUILD_METHOD = "morton"
    MORTON_BITS = 10

    def __init__(self):
        self.nodes = _NodeView(length=0)
        self.ordered_tris = np.zeros(0, np.int32)
        self.mat_palette = []
        self._mat_key_to_idx = {}
        self._batch = TriangleBatch.empty()
        self._source_mat_idx = np.zeros(0, np.int32)
        self.native = None
        self.method = None
        self._set_ordered(np.zeros(0, np.int32))

    @property
    def triangle_count(self):
        return len(self.ordered_tris)

    # -- host-side preparation ------------------------------------------------
    @staticmethod
    def _coerce_batches(tri_data):
        if isinstance(tri_data, TriangleBatch):
            return [tri_data]
        if not tri_data:
            return []
        if all(isinstance(b, TriangleBatch) for b in tri_data):
            return list(tri_data)
        return [TriangleBatch.from_dicts(tri_data)]

    def _add_material(self, rec):
        key = (int(rec.get("mat_type", rec.get("type"))), tuple(float(v) for v in rec["albedo"]),
               float(rec["roughness"]), float(rec["ior"]), float(rec["emission"]), int(rec.get("texture_idx", -1)))
        if key not in self._mat_key_to_idx:
            self._mat_key_to_idx[key] = len(self.mat_palette)
            self.mat_palette.append({"type": key[0], "albedo": list(key[1]), "roughness": key[2], "ior": key[3],
                                     "emission": key[4], "texture_idx": key[5]})
        return self._mat_key_to_idx[key]

    def _material_indices(self, batch):
        if batch.mat_idx is not None:
            remap = np.array([self._add_material(m) for m in batch.mat_palette] or [0], np.int32)
            return remap[batch.mat_idx] if batch.triangle_count else np.zeros(0, np.int32)
        # per-triangle materials: unique rows in first-seen order
        rows = np.concatenate([batch.mat_type[:, None].astype(np.float64), batch.albedo.astype(np.float64),
                               batch.roughness[:, None].astype(np.float64), batch.ior[:, None].astype(np.float64),
                               batch.emission[:, None].astype(np.float64),
                               batch.texture_idx[:, None].astype(np.float64)], axis=1)
        uniq, first, inv = np.unique(rows, axis=0, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")
        remap = np.zeros(len(uniq), np.int32)
        for j in order:
            r = uniq[j]
            remap[j] = self._add_material({"mat_type": int(r[0]), "albedo": r[1:4].tolist(), "roughness": r[4],
                                           "ior": r[5], "emission": r[6], "texture_idx": int(r[7])})
        return remap[inv.reshape(-1)]

    def _set_ordered(self, order):
        b = self._batch
        self.ordered_tris = np.asarray(order, np.int32)
        o = self.ordered_tris
        self._ordered_v0, self._ordered_v1, self._ordered_v2 = b.v0[o], b.v1[o], b.v2[o]
        self._ordered_n0, self._ordered_n1, self._ordered_n2 = b.n0[o], b.n1[o], b.n2[o]
        self._ordered_uv0, self._ordered_uv1, self._ordered_uv2 = b.uv0[o], b.uv1[o], b.uv2[o]
        self._ordered_has_uv = b.has_uv[o]
        self._ordered_mat_idx = (self._source_mat_idx[o] if len(self._source_mat_idx)
                                 else np.zeros(len(o), np.int32))

    def palette_arrays(self):
        pal = self.mat_palette or [{"type": 0, "albedo": [0.8, 0.8, 0.8], "roughness": 0.0, "ior": 1.0,
                                    "emission": 0.0}]
        return (np.array([m["type"] for m in pal], np.int32), np.array([m["albedo"] for m in pal], np.float32),
                np.array([m["roughness"] for m in pal], np.float32), np.array([m["ior"] for m in pal], np.float32),
                np.array([m["emission"] for m in pal], np.float32))

    def palette_textures(self):
        """Texture index of each palette entry (-1: untextured)."""
        pal = self.mat_palette or [{}]
        return np.array([int(m.get("texture_idx", -1)) for m in pal], np.int32)

    # -- build ------------------------------------------------------------------
    def build(self, tri_data, method=None, native=None):
        """Build from TriangleBatch objects or legacy triangle dicts."""
        batch = TriangleBatch.concat(self._coerce_batches(tri_data))
        self._batch = batch
        self.mat_palette = []
        self._mat_key_to_idx = {}
        self._source_mat_idx = self._material_indices(batch) if batch.triangle_count else np.zeros(0, np.int32)
        method = method or self.BUILD_METHOD
        if method not in ("morton", "median", "lbvh"):
            raise ValueError(f"Unknown BVH build method: {method}")
        self.method = method
        self.native = native or nat.NativeScene()
        sc = self.native
        sc.set_triangles(batch.v0, batch.v1, batch.v2, batch.n0, batch.n1, batch.n2, self._source_mat_idx)
        sc.set_materials(*self.palette_arrays())
        if batch.triangle_count == 0:
            self.nodes = _NodeView(length=0)
            self._set_ordered(np.zeros(0, np.int32))
            return self
        if method == "morton":
            sc.build_bvh(nat.RX_BVH_REFERENCE, int(self.MAX_LEAF_SIZE))
            arrays = sc.export_reference()
            self.nodes = _NodeView(arrays)
            self._set_ordered(arrays["order"])
        elif method == "median":
            arrays = self._median_tree(batch)
            sc.set_reference_bvh(arrays["node_min"], arrays["node_max"], arrays["left"], arrays["right"],
                                 arrays["start"], arrays["count"], arrays["order"])
            self.nodes = _NodeView(arrays)
            self._set_ordered(arrays["order"])
        else:
            sc.build_bvh(nat.RX_BVH_LBVH_SAH, min(int(self.MAX_LEAF_SIZE), 15), True)
            info = sc.bvh_info()
            self.nodes = _NodeView(length=info["n_nodes"])
            self._set_ordered(np.arange(batch.triangle_count, dtype=np.int32))
        return self

    def _median_tree(self, batch):
        """Longest-axis median split of the reference's legacy method
        (bvh_builder.py:488-525) on the host."""
        eps = np.float32(1e-4)
        stacked = np.stack([batch.v0, batch.v1, batch.v2], axis=1)
        bmin, bmax = stacked.min(axis=1) - eps, stacked.max(axis=1) + eps
        cen = (batch.v0 + batch.v1 + batch.v2) / np.float32(3.0)
        nodes, chunks = [], []
        count = [0]

        def rec(idx, depth):
            me = len(nodes)
            nodes.append(None)
            lo, hi = bmin[idx].min(axis=0), bmax[idx].max(axis=0)
            if len(idx) <= self.MAX_LEAF_SIZE or depth >= self.MAX_DEPTH:
                nodes[me] = (lo, hi, -1, -1, count[0], len(idx))
                chunks.append(idx)
                count[0] += len(idx)
            else:
                axis = self._longest_axis(lo, hi)
                mid = len(idx) // 2
                part = idx[np.argpartition(cen[idx, axis], mid)]
                left = rec(part[:mid], depth + 1)
                right = rec(part[mid:], depth + 1)
                nodes[me] = (lo, hi, left, right, -1, 0)
            return me

        rec(np.arange(batch.triangle_count, dtype=np.int32), 0)
        return {"node_min": np.array([n[0] for n in nodes], np.float32),
                "node_max": np.array([n[1] for n in nodes], np.float32),
                "left": np.array([n[2] for n in nodes], np.int32), "right": np.array([n[3] for n in nodes], np.int32),
                "start": np.array([n[4] for n in nodes], np.int32), "count": np.array([n[5] for n in nodes], np.int32),
                "order": np.concatenate(chunks).astype(np.int32)}

    @staticmethod
    def _longest_axis(aabb_min, aabb_max):
        ex, ey, ez = np.asarray(aabb_max) - np.asarray(aabb_min)
        if ex >= ey and ex >= ez:
            return 0
        if ey >= ez:
            return 1
        return 2

    def upload(self):
        """Make this tree the one `render_kernel` traces (the reference copies
        it into global fields; here it is already resident on the device)."""
        from rendering.taichi import fields
        fields.bind_builder(self)
        return self
