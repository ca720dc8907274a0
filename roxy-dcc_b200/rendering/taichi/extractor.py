"""extract_scene: scene graph -> device scene (rendering/taichi/extractor.py).

Flattens World objects the way the reference does — Mesh triangles and
IndexedMesh arrays in world space into one triangle set with a material
palette, analytic primitives into object slots, albedo textures into an
indexed table — but in vectorised numpy and one upload per array instead
of per-element field stores.  The renderer's path ("lbvh") transforms
IndexedMesh geometry on the device; the BVH is built on the GPU.
"""
import numpy as np

import roxy_native as nat
from rendering.taichi.bvh_builder import GPUBVHBuilder, TriangleBatch
from rendering.taichi.lights import build_lights

_DEFAULT_ALBEDO = (0.8, 0.8, 0.8)
MAX_TEXTURES = 8
MAX_TEXTURE_SIZE = 2048


class TextureTable:
    """Albedo textures in the order extract_scene numbers them
    (extractor.py:96-117): first use in visit order, keyed by (path, flip_v,
    identity of an in-memory texture)."""

    def __init__(self):
        self.textures = []
        self._index = {}

    def index(self, mat):
        tex = getattr(mat, "_albedo_texture", None)
        if tex is None:
            return -1
        key = (tex.path, bool(tex.flip_v), id(tex) if tex.path is None else None)
        if key not in self._index:
            if len(self.textures) >= MAX_TEXTURES:
                raise ValueError(f"Scene has more than {MAX_TEXTURES} image textures; "
                                 "increase MAX_TEXTURES in rendering/taichi/fields.py")
            self._index[key] = len(self.textures)
            self.textures.append(tex)
        return self._index[key]

    def images(self):
        """(uint8 HxWx3 images, flip_v flags) as _upload_textures stores them."""
        imgs = []
        for t in self.textures:
            data = np.asarray(t.load_pixels_u8(max_size=MAX_TEXTURE_SIZE), dtype=np.uint8)
            if data.shape[0] > MAX_TEXTURE_SIZE or data.shape[1] > MAX_TEXTURE_SIZE:
                raise ValueError(f"texture of {data.shape[1]}x{data.shape[0]} exceeds {MAX_TEXTURE_SIZE}")
            imgs.append(data[:, :, :3])
        return imgs, [1 if t.flip_v else 0 for t in self.textures]

    def __len__(self):
        return len(self.textures)


def _mat_record(mat, textures=None):
    from scene.scene_object import SceneObject
    if mat is None:
        return {"mat_type": 0, "albedo": list(_DEFAULT_ALBEDO), "roughness": 0.0, "ior": 1.0, "emission": 0.0,
                "texture_idx": -1}
    r = SceneObject.material_record(mat)
    r["texture_idx"] = textures.index(mat) if textures is not None else -1
    return r


def _xform_points(M, pts):
    """Row-by-row `M.transform_point` with the same double-precision order."""
    r = M.rows
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    X = x * r[0][0] + y * r[0][1] + z * r[0][2] + r[0][3]
    Y = x * r[1][0] + y * r[1][1] + z * r[1][2] + r[1][3]
    Z = x * r[2][0] + y * r[2][1] + z * r[2][2] + r[2][3]
    W = x * r[3][0] + y * r[3][1] + z * r[3][2] + r[3][3]
    out = np.stack([X, Y, Z], axis=1)
    nz = W != 0
    out[nz] = out[nz] / W[nz, None]
    return out


def _xform_normals(M, nrm):
    """`inv_T.transform_vector(n).normalize()` per row (v * (1 / |v|))."""
    r = M.rows
    x, y, z = nrm[:, 0], nrm[:, 1], nrm[:, 2]
    X = x * r[0][0] + y * r[0][1] + z * r[0][2]
    Y = x * r[1][0] + y * r[1][1] + z * r[1][2]
    Z = x * r[2][0] + y * r[2][1] + z * r[2][2]
    length = np.sqrt(X * X + Y * Y + Z * Z)
    inv = np.where(length > 0, 1.0 / np.where(length > 0, length, 1.0), 0.0)
    return np.stack([X * inv, Y * inv, Z * inv], axis=1)


def _mesh_batch(obj, shape, mesh, textures=None):
    tris = mesh._triangles
    if not tris:
        return None
    M = obj.world_matrix
    inv_T = obj.world_inverse_transpose_matrix
    n = len(tris)
    V = np.empty((n, 3, 3), np.float64)
    N = np.empty((n, 3, 3), np.float64)
    UV = np.zeros((n, 3, 2), np.float64)
    has_uv = np.zeros(n, np.int32)
    groups = {}
    mat_idx = np.empty(n, np.int32)
    recs = []
    for i, t in enumerate(tris):
        V[i, 0], V[i, 1], V[i, 2] = tuple(t._v0), tuple(t._v1), tuple(t._v2)
        f = t._normal
        N[i, 0] = tuple(t._n0 if t._n0 is not None else f)
        N[i, 1] = tuple(t._n1 if t._n1 is not None else f)
        N[i, 2] = tuple(t._n2 if t._n2 is not None else f)
        if t._uv0 is not None and t._uv1 is not None and t._uv2 is not None:
            UV[i, 0], UV[i, 1], UV[i, 2] = tuple(t._uv0), tuple(t._uv1), tuple(t._uv2)
            has_uv[i] = 1
        g = t._group
        if g not in groups:
            groups[g] = len(recs)
            recs.append(_mat_record(shape.material_for_group(g), textures))
        mat_idx[i] = groups[g]
    Vw = _xform_points(M, V.reshape((-1, 3))).reshape((n, 3, 3)).astype(np.float32)
    Nw = _xform_normals(inv_T, N.reshape((-1, 3))).reshape((n, 3, 3)).astype(np.float32)
    k = len(recs)
    return TriangleBatch(Vw[:, 0], Vw[:, 1], Vw[:, 2], Nw[:, 0], Nw[:, 1], Nw[:, 2],
                         np.array([r["mat_type"] for r in recs], np.int32).reshape(k),
                         np.array([r["albedo"] for r in recs], np.float32).reshape((k, 3)),
                         np.array([r["roughness"] for r in recs], np.float32).reshape(k),
                         np.array([r["ior"] for r in recs], np.float32).reshape(k),
                         np.array([r["emission"] for r in recs], np.float32).reshape(k),
                         uv0=UV[:, 0], uv1=UV[:, 1], uv2=UV[:, 2], has_uv=has_uv,
                         texture_idx=np.array([r["texture_idx"] for r in recs], np.int32).reshape(k),
                         mat_idx=mat_idx)


def _walk(world):
    """Renderable geometry in visit order: ("mesh" | "indexed", object, shape,
    geometry) items and the object-slot dicts of analytic primitives."""
    from scene.mesh import IndexedMesh, Mesh
    items, slots = [], []

    def visit(obj):
        if not obj.renderable:
            return
        for shape in obj.shapes:
            geo = shape.geometry
            if isinstance(geo, Mesh):
                items.append(("mesh", obj, shape, geo))
            elif isinstance(geo, IndexedMesh):
                items.append(("indexed", obj, shape, geo))
            else:
                exported = obj.taichi_export()
                if isinstance(exported, list):
                    slots.extend(exported)
                elif exported:
                    slots.append(exported)
                break
        for child in obj.children:
            visit(child)

    for o in world.objects:
        visit(o)
    return items, slots


def _group_records(shape, geo, textures):
    """Material record of every group of an IndexedMesh, in group order."""
    return {gi: _mat_record(shape.material_for_group(g), textures) for gi, g in enumerate(geo.groups)}


def collect(world, textures=None):
    """(triangle batches, object slots) of every renderable object.  IndexedMesh
    batches come first in visit order and Mesh triangles after them, the
    order extract_scene gives the reference's builder; `textures` (a
    TextureTable) receives the albedo textures in the reference's order."""
    items, slots = _walk(world)
    indexed, meshes = [], []
    for kind, obj, shape, geo in items:
        if kind == "indexed":
            arrays = geo.indexed_triangle_arrays(obj.world_matrix, obj.world_inverse_transpose_matrix)
            indexed.append(TriangleBatch.from_indexed_arrays(arrays, _group_records(shape, geo, textures)))
        else:
            b = _mesh_batch(obj, shape, geo, textures)
            if b is not None:
                meshes.append(b)
    return indexed + meshes, slots


def slot_arrays(slots):
    n = len(slots)
    z3 = [0.0, 0.0, 0.0]
    g = lambda k, d: [s.get(k, d) for s in slots]  # noqa: E731
    return {"type": np.array(g("type", 0), np.int32).reshape(n),
            "center": np.array(g("center", z3), np.float32).reshape((n, 3)),
            "radius": np.array(g("radius", 0.0), np.float32).reshape(n),
            "normal": np.array(g("normal", z3), np.float32).reshape((n, 3)),
            "offset": np.array(g("offset", 0.0), np.float32).reshape(n),
            "extra": np.array(g("extra", z3), np.float32).reshape((n, 3)),
            "v0": np.array(g("v0", z3), np.float32).reshape((n, 3)),
            "v1": np.array(g("v1", z3), np.float32).reshape((n, 3)),
            "v2": np.array(g("v2", z3), np.float32).reshape((n, 3)),
            "mat_type": np.array(g("mat_type", 0), np.int32).reshape(n),
            "albedo": np.array(g("albedo", z3), np.float32).reshape((n, 3)),
            "roughness": np.array(g("roughness", 0.0), np.float32).reshape(n),
            "ior": np.array(g("ior", 1.0), np.float32).reshape(n),
            "emission": np.array(g("emission", 0.0), np.float32).reshape(n)}


class DeviceScene:
    """Everything the renderer needs for one world: the native scene (with its
    BVH), object slots and both light lists.

    light_args: (v0, v1, v2, palette index) of at least every emissive
    triangle, in scene order, followed by the palette's type, albedo and
    emission arrays; light_index: scene triangle index of each of those rows
    (None: the rows are all triangles in scene order); pal_texture: texture
    index per palette entry.
    h2d_bytes: bytes copied host -> device for the geometry."""

    def __init__(self, native, slots, stats, light_args, builder=None, h2d_bytes=0, pal_texture=None,
                 light_index=None):
        self.native = native
        self.slots = slots
        self.stats = stats
        self.builder = builder
        self.h2d_bytes = int(h2d_bytes)
        self._light_args = light_args
        self._light_index = light_index
        self.pal_texture = pal_texture
        self._lights_mode = None

    @classmethod
    def from_builder(cls, builder, slots, stats, h2d_extra=0):
        b = builder._batch
        pal = builder.palette_arrays()
        h2d = sum(a.nbytes for a in (b.v0, b.v1, b.v2, b.n0, b.n1, b.n2)) + 4 * b.triangle_count + h2d_extra
        return cls(builder.native, slots, stats, (b.v0, b.v1, b.v2, builder._source_mat_idx, pal[0], pal[1], pal[4]),
                   builder=builder, h2d_bytes=h2d, pal_texture=builder.palette_textures())

    def use_lights(self, compat):
        compat = bool(compat)
        if self._lights_mode is compat:
            return
        lights = build_lights(self.slots, *self._light_args, compat=compat, pal_texture=self.pal_texture,
                              tri_index=self._light_index)
        self.native.set_lights(lights)
        self._lights_mode = compat


class HostScene:
    """Host-side flattening of a world: concatenated triangles, palette,
    per-triangle palette index, object slots and textures (no device work)."""

    def __init__(self, world):
        self.texture_table = TextureTable()
        batches, slots = collect(world, self.texture_table)
        self.batches = batches
        self.slots = slots
        self.batch = TriangleBatch.concat(batches)
        self.builder = GPUBVHBuilder()
        self.mat_idx = (self.builder._material_indices(self.batch) if self.batch.triangle_count
                        else np.zeros(0, np.int32))
        self.palette = self.builder.palette_arrays()
        self.mat_texture = self.builder.palette_textures()
        self.textures, self.tex_flip = self.texture_table.images()

    def lights(self, compat):
        b = self.batch
        return build_lights(self.slots, b.v0, b.v1, b.v2, self.mat_idx, self.palette[0], self.palette[1],
                            self.palette[4], compat=compat, pal_texture=self.mat_texture)


def _indexed_world_positions(geo, matrix, sel):
    """float32 world-space corners (len(sel), 3, 3) of triangles `sel` of an
    IndexedMesh, in the element-wise float64 order of k_extract_indexed."""
    p = geo._positions[geo._tri_pos_idx[sel]]
    if matrix is None:
        return p.astype(np.float32)
    r = np.asarray(matrix.rows, dtype=np.float64)
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    out = np.stack([((x * r[i, 0] + y * r[i, 1]) + z * r[i, 2]) + r[i, 3] for i in range(3)], axis=-1)
    w = ((x * r[3, 0] + y * r[3, 1]) + z * r[3, 2]) + r[3, 3]
    div = np.abs(w) > 1e-12
    out[div] = out[div] / w[div][:, None]
    return out.astype(np.float32)


def _emissive(builder, palette_idx):
    m = builder.mat_palette[int(palette_idx)]
    return m["type"] == 3 and m["emission"] > 0.0


def _textured(builder, palette_idx):
    return builder.mat_palette[int(palette_idx)].get("texture_idx", -1) >= 0


def _extract_on_device(world, native, builder, textures):
    """Fill `native`'s triangle arrays with the world's triangles in the order
    and palette of collect() + GPUBVHBuilder.build, transforming IndexedMesh
    geometry on the device (rx_scene_put_indexed).  Returns (slots, triangle
    count, emissive triangle rows, host->device bytes, scene triangle index of
    each emissive row)."""
    items, slots = _walk(world)
    # material records in visit order (this numbers the textures as the
    # reference does), then triangles: IndexedMesh first, Mesh after
    indexed, mesh_batches = [], []
    for kind, obj, shape, geo in items:
        if kind == "indexed":
            indexed.append((obj, geo, _group_records(shape, geo, textures)))
        else:
            b = _mesh_batch(obj, shape, geo, textures)
            if b is not None:
                mesh_batches.append(b)
    total = sum(g.triangle_count for _, g, _ in indexed) + sum(b.triangle_count for b in mesh_batches)
    native.alloc_triangles(total)
    lv0, lv1, lv2, lmat, lidx = [], [], [], [], []
    off, h2d = 0, 0
    for obj, geo, recs in indexed:
        n = geo.triangle_count
        if n == 0:
            continue
        groups = geo.groups
        gidx = geo._tri_group_idx
        lo, hi = int(gidx.min()), int(gidx.max())
        if lo < 0 or hi >= len(groups):
            raise ValueError("IndexedMesh group index outside its group list")
        # the groups in use, ascending; a mesh of one group needs no count
        used = np.array([lo]) if lo == hi else np.nonzero(np.bincount(gidx, minlength=len(groups)))[0]
        group_mat = np.zeros(len(groups), np.int32)
        for g in used:
            group_mat[g] = builder._add_material(TriangleBatch.palette_record(recs[int(g)]))
        has_n = geo._normals is not None
        native.put_indexed(off, geo._positions, geo._tri_pos_idx, geo._normals if has_n else None,
                           geo._tri_normal_idx if has_n else None, obj.world_matrix.rows,
                           obj.world_inverse_transpose_matrix.rows, gidx, group_mat)
        h2d += geo._positions.nbytes + geo._tri_pos_idx.nbytes + gidx.nbytes + group_mat.nbytes
        if has_n:
            h2d += geo._normals.nbytes + geo._tri_normal_idx.nbytes
        if any(_textured(builder, group_mat[g]) for g in used):
            uv = geo.indexed_uv_arrays()
            native.put_uvs(off, uv["uv0"], uv["uv1"], uv["uv2"], uv["has_uv"])
            h2d += sum(a.nbytes for a in uv.values())
        em = [g for g in used if _emissive(builder, group_mat[g])]
        if em:
            sel = np.nonzero(np.isin(gidx, em))[0]
            w = _indexed_world_positions(geo, obj.world_matrix, sel)
            lv0.append(w[:, 0])
            lv1.append(w[:, 1])
            lv2.append(w[:, 2])
            lmat.append(group_mat[gidx[sel]])
            lidx.append(off + sel)
        off += n
    for b in mesh_batches:
        remap = np.array([builder._add_material(m) for m in b.mat_palette], np.int32)
        mat = remap[b.mat_idx]
        native.put_triangles(off, b.v0, b.v1, b.v2, b.n0, b.n1, b.n2, mat)
        h2d += sum(a.nbytes for a in (b.v0, b.v1, b.v2, b.n0, b.n1, b.n2)) + mat.nbytes
        if any(_textured(builder, k) for k in remap):
            native.put_uvs(off, b.uv0, b.uv1, b.uv2, b.has_uv)
            h2d += sum(a.nbytes for a in (b.uv0, b.uv1, b.uv2, b.has_uv))
        sel = np.nonzero([_emissive(builder, k) for k in remap])[0]
        if len(sel):
            rows = np.nonzero(np.isin(b.mat_idx, sel))[0]
            lv0.append(b.v0[rows])
            lv1.append(b.v1[rows])
            lv2.append(b.v2[rows])
            lmat.append(mat[rows])
            lidx.append(off + rows)
        off += b.triangle_count
    cat3 = lambda xs: np.concatenate(xs) if xs else np.zeros((0, 3), np.float32)  # noqa: E731
    lights = (cat3(lv0), cat3(lv1), cat3(lv2), np.concatenate(lmat) if lmat else np.zeros(0, np.int32))
    light_index = np.concatenate(lidx).astype(np.int32) if lidx else np.zeros(0, np.int32)
    return slots, total, lights, h2d, light_index


def _upload_textures(native, builder, textures):
    """Texture images and the palette's texture indices; bytes copied."""
    if not len(textures):
        return 0
    imgs, flips = textures.images()
    native.set_textures(imgs, flips)
    native.set_material_textures(builder.palette_textures())
    return sum(im.nbytes for im in imgs)


def build_device_scene(world, method="lbvh", leaf_size=None, ctx=None):
    """Extract `world` to a device scene with a BVH.  method "lbvh" (the
    renderer's) transforms IndexedMesh geometry on the device; "morton" and
    "median" go through GPUBVHBuilder's host flattening so that the
    reference-format tree and ordered arrays stay available.  `ctx`: the
    context (device stream) that builds it, by default the device's shared
    one; a scene built on another context of the same device can be
    rendered and served by any of them once that context is synchronised."""
    textures = TextureTable()
    if method != "lbvh":
        batches, slots = collect(world, textures)
        builder = GPUBVHBuilder()
        if leaf_size is not None:
            builder.MAX_LEAF_SIZE = leaf_size
        native = nat.NativeScene(ctx)
        native.set_objects(slot_arrays(slots) if slots else None)
        builder.build(batches, method=method, native=native)
        h2d = _upload_textures(native, builder, textures)
        b = builder._batch
        if h2d and b.triangle_count:
            native.put_uvs(0, b.uv0, b.uv1, b.uv2, b.has_uv)
        stats = {"primitive_count": len(slots), "bvh_nodes": len(builder.nodes),
                 "bvh_triangles": builder.triangle_count,
                 "bvh_materials": len(builder.mat_palette) if batches else 0,
                 "bvh_leaf_size": builder.MAX_LEAF_SIZE if builder.triangle_count else 0}
        return DeviceScene.from_builder(builder, slots, stats, h2d_extra=h2d)
    leaf = 4 if leaf_size is None else int(leaf_size)
    native = nat.NativeScene(ctx)
    builder = GPUBVHBuilder()  # palette bookkeeping only
    slots, total, light_tris, h2d, light_index = _extract_on_device(world, native, builder, textures)
    native.set_objects(slot_arrays(slots) if slots else None)
    pal = builder.palette_arrays()
    native.set_materials(*pal)
    h2d += _upload_textures(native, builder, textures)
    n_nodes = 0
    if total:
        native.build_bvh(nat.RX_BVH_LBVH_SAH, min(leaf, 15), True)
        n_nodes = native.bvh_info()["n_nodes"]
    stats = {"primitive_count": len(slots), "bvh_nodes": n_nodes, "bvh_triangles": total,
             "bvh_materials": len(builder.mat_palette), "bvh_leaf_size": leaf if total else 0}
    return DeviceScene(native, slots, stats, light_tris + (pal[0], pal[1], pal[4]), h2d_bytes=h2d,
                       pal_texture=builder.palette_textures(), light_index=light_index)


def extract_scene(world, method="lbvh"):
    """Extract `world` to the device and make it the scene `render_kernel`
    traces.  Returns the reference's stats dict."""
    from rendering.taichi import fields
    ds = build_device_scene(world, method=method)
    fields.bind_scene(ds)
    return dict(ds.stats)
