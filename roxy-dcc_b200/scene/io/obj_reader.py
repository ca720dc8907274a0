"""Wavefront OBJ reader with the reference's interface
(scene/io/obj_reader.py:124-646: OBJReader.load / load_as_mesh /
load_as_indexed_mesh / _parse_indexed / _load_python_indexed /
_load_python).

The text is parsed on the GPU (rx_obj_* in libroxy_cuda.so): line split,
keyword classification, exact float64 conversion and fan triangulation run
one thread per line over the whole file.  The host reads only the lines the
device lists: usemtl / mtllib / o / g (the structure), unrecognised tokens
(the reference's warning), and the rare lines whose numbers the device does
not convert exactly or that hold non-ASCII bytes; those are parsed here with
the reference's own rules (str.split, float(), int()), so results and
exceptions are the reference's.  There is no CPU fallback for the bulk of
the file: without the CUDA library the reader raises.
"""
import ctypes
import time
from pathlib import Path

import numpy as np

import roxy_native as nat
from core import Color, Vec2, Vec3
from scene.materials import Diffuse
from scene.mesh import IndexedMesh, Mesh, Triangle

_KIND = {"v": nat.RX_OBJ_V, "vn": nat.RX_OBJ_VN, "vt": nat.RX_OBJ_VT, "f": nat.RX_OBJ_F,
         "usemtl": nat.RX_OBJ_USEMTL, "mtllib": nat.RX_OBJ_MTLLIB, "o": nat.RX_OBJ_O, "g": nat.RX_OBJ_G,
         "s": nat.RX_OBJ_S}
# per-line counts the device scans: v, vn, vt, triangles, usemtl, faces
_PV, _PVN, _PVT, _PTRI, _PMTL, _PFACE = range(6)


def _line_kind(parts):
    if not parts or parts[0].startswith("#"):
        return nat.RX_OBJ_SKIP
    return _KIND.get(parts[0], nat.RX_OBJ_OTHER)


def _idx(raw, length):
    i = int(raw)
    return i - 1 if i > 0 else length + i


def _face_indices(face, lv, lvt, lvn):
    """vi / uvi / ni of one face's vertex tokens (obj_reader.py:405-411)."""
    vi, ni, uvi = [], [], []
    for part in face:
        vals = part.split("/")
        vi.append(_idx(vals[0], lv))
        uvi.append(_idx(vals[1], lvt) if len(vals) > 1 and vals[1] else -1)
        ni.append(_idx(vals[2], lvn) if len(vals) > 2 and vals[2] else -1)
    return vi, uvi, ni


class ObjData:
    """One parsed OBJ text: shared float64 arrays, per-triangle int32 index
    tables in file order, the usemtl group names, and the structural
    events (usemtl / mtllib / o / g) with the counts before each."""

    def __init__(self):
        self.positions = self.normals = self.uvs = None
        self.tri_pos_idx = self.tri_normal_idx = self.tri_uv_idx = self.tri_group_idx = None
        self.group_names = ["default"]
        self.events = []  # (keyword, parts, counts before the line: v, vn, vt, tri, usemtl, faces)
        self.lines = 0
        self.totals = np.zeros(7, np.int32)  # v, vn, vt, tri, usemtl, faces, listed
        self.device_ms = 0.0  # kernel time of the parse (CUDA events)

    triangle_count = property(lambda s: len(s.tri_pos_idx))


def parse_obj_bytes(data, ctx=None):
    """Parse OBJ text (bytes) on the GPU; see the module docstring."""
    ctx = ctx or nat.context()
    L = nat.lib()
    buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
    h = ctypes.c_void_p()
    lines, listed = ctypes.c_int(), ctypes.c_int()
    ctx.check(L.rx_obj_begin(ctx.h, ctypes.c_void_p(buf.ctypes.data), len(data), ctypes.byref(h),
                             ctypes.byref(lines), ctypes.byref(listed)))
    try:
        return _finish(ctx, L, h, data, lines.value, listed.value)
    finally:
        L.rx_obj_end(h)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


def _finish(ctx, L, h, data, n_lines, n_listed):
    out = ObjData()
    out.lines = n_lines
    off = np.zeros(n_listed, np.int64)
    length = np.zeros(n_listed, np.int32)
    kind = np.zeros(n_listed, np.int32)
    flags = np.zeros(n_listed, np.int32)
    if n_listed:
        ctx.check(L.rx_obj_listed(h, _ptr(off), _ptr(length), _ptr(kind), _ptr(flags), None))
    # the listed lines as text (the reference reads the file as UTF-8 text;
    # only listed lines can hold non-ASCII bytes, so a decoding error
    # surfaces here as it would there)
    texts = [data[o:o + n].decode("utf-8") for o, n in zip(off.tolist(), length.tolist())]
    parts_of = [t.split() for t in texts]
    # kinds and triangle counts of non-ASCII lines as Python splits them
    fix = [i for i in range(n_listed) if flags[i] & nat.RX_OBJ_NONASCII]
    if fix:
        pos = np.asarray(fix, np.int32)
        k_new = np.asarray([_line_kind(parts_of[i]) for i in fix], np.int32)
        t_new = np.asarray([max(0, len(parts_of[i]) - 3) if k == nat.RX_OBJ_F else 0
                            for i, k in zip(fix, k_new.tolist())], np.int32)
        kind[pos] = k_new
        ctx.check(L.rx_obj_correct(h, len(fix), _ptr(pos), _ptr(k_new), _ptr(t_new)))
    totals = np.zeros(7, np.int32)
    prefix = np.zeros((max(n_listed, 1), 6), np.int32)
    ctx.check(L.rx_obj_scan(h, _ptr(totals), _ptr(prefix)))
    out.totals = totals

    # structure and host-parsed values, in file order
    group_to_idx = {"default": 0}
    usemtl_gid = []
    current_gid = 0
    host_v, host_f = [], []
    for i in range(n_listed):
        k, parts, pre = int(kind[i]), parts_of[i], prefix[i]
        if k == nat.RX_OBJ_SKIP or k == nat.RX_OBJ_S:
            continue
        if k == nat.RX_OBJ_USEMTL:
            name = parts[1] if len(parts) > 1 else "default"
            if name not in group_to_idx:
                group_to_idx[name] = len(out.group_names)
                out.group_names.append(name)
            current_gid = group_to_idx[name]
            usemtl_gid.append(current_gid)
            out.events.append(("usemtl", parts, pre))
        elif k in (nat.RX_OBJ_MTLLIB, nat.RX_OBJ_O, nat.RX_OBJ_G):
            out.events.append((parts[0], parts, pre))
        elif k == nat.RX_OBJ_OTHER:
            print(f"Warning: Unrecognized OBJ token: {parts[0]!r}")
        elif flags[i] & nat.RX_OBJ_HOST:
            if k == nat.RX_OBJ_V:
                host_v.append(("v", int(pre[_PV]), [float(parts[1]), float(parts[2]), float(parts[3])]))
            elif k == nat.RX_OBJ_VN:
                host_v.append(("vn", int(pre[_PVN]), [float(parts[1]), float(parts[2]), float(parts[3])]))
            elif k == nat.RX_OBJ_VT:
                host_v.append(("vt", int(pre[_PVT]), [float(parts[1]), float(parts[2])]))
            elif k == nat.RX_OBJ_F:
                vi, uvi, ni = _face_indices(parts[1:], int(pre[_PV]), int(pre[_PVT]), int(pre[_PVN]))
                host_f.append((int(pre[_PTRI]), vi, uvi, ni, current_gid))

    nv, nvn, nvt, nt = (int(x) for x in totals[:4])
    out.positions = np.zeros((nv, 3), np.float64)
    out.normals = np.zeros((nvn, 3), np.float64)
    out.uvs = np.zeros((nvt, 2), np.float64)
    out.tri_pos_idx = np.zeros((nt, 3), np.int32)
    out.tri_normal_idx = np.zeros((nt, 3), np.int32)
    out.tri_uv_idx = np.zeros((nt, 3), np.int32)
    out.tri_group_idx = np.zeros(nt, np.int32)
    gid = np.asarray(usemtl_gid if usemtl_gid else [0], np.int32)
    ctx.check(L.rx_obj_emit(h, _ptr(gid), _ptr(out.positions), _ptr(out.normals), _ptr(out.uvs),
                            _ptr(out.tri_pos_idx), _ptr(out.tri_normal_idx), _ptr(out.tri_uv_idx),
                            _ptr(out.tri_group_idx)))
    dst = {"v": out.positions, "vn": out.normals, "vt": out.uvs}
    for key, row, vals in host_v:
        dst[key][row] = vals
    for t0, vi, uvi, ni, g in host_f:
        for j in range(1, len(vi) - 1):
            t = t0 + j - 1
            out.tri_pos_idx[t] = (vi[0], vi[j], vi[j + 1])
            out.tri_uv_idx[t] = (uvi[0], uvi[j], uvi[j + 1])
            out.tri_normal_idx[t] = (ni[0], ni[j], ni[j + 1])
            out.tri_group_idx[t] = g
    ms = ctypes.c_float()
    ctx.check(L.rx_obj_device_ms(h, ctypes.byref(ms)))
    out.device_ms = ms.value
    return out


def parse_obj(path, ctx=None):
    return parse_obj_bytes(Path(path).read_bytes(), ctx)


class _Progress:
    """The reference's progress callbacks (obj_reader.py:29-119), emitted at
    the phase boundaries of the device parse."""

    def __init__(self, callback):
        self._cb = callback
        self.object_name = ""
        self.group_name = ""
        self.material_name = "default"

    def emit(self, phase, detail):
        if self._cb:
            self._cb(phase, detail)

    def detail(self, d, percent=100.0):
        t = d.totals
        labels = []
        if self.object_name:
            labels.append(f"object: {self.object_name}")
        if self.group_name:
            labels.append(f"group: {self.group_name}")
        if self.material_name:
            labels.append(f"material: {self.material_name}")
        suffix = " • ".join(labels)
        if suffix:
            suffix = " • " + suffix
        return (f"{percent:5.1f}% • {d.lines:,} lines • {int(t[0]):,} verts • {int(t[2]):,} uvs • "
                f"{int(t[5]):,} faces • {int(t[3]):,} tris{suffix}")

    def track(self, d):
        for key, parts, _ in d.events:
            if key == "o":
                self.object_name = parts[1] if len(parts) > 1 else "object"
            elif key == "g":
                self.group_name = parts[1] if len(parts) > 1 else "group"
            elif key == "usemtl":
                self.material_name = parts[1] if len(parts) > 1 else "default"


def _default_material():
    return Diffuse(Color(0.8, 0.8, 0.8))


def _load_mtllib(file_path, parts, progress=None):
    """{name: Material} of an mtllib line's file, None when it does not exist."""
    from scene.io.mtl_loader import MTLLoader
    mtl_path = file_path.parent / parts[1]
    if progress:
        progress.emit("Loading material library", str(mtl_path))
    if mtl_path.exists():
        raw = MTLLoader.load(str(mtl_path))
        return {n: m.to_material() for n, m in raw.items()}
    return None


def _tri_ranges_used(d):
    """Names of the usemtl groups that received triangles (obj_reader.py:417)."""
    used = set()
    mtl, start = "default", 0
    for key, parts, pre in d.events:
        if key != "usemtl":
            continue
        if int(pre[_PTRI]) > start:
            used.add(mtl)
        mtl, start = (parts[1] if len(parts) > 1 else "default"), int(pre[_PTRI])
    if d.triangle_count > start:
        used.add(mtl)
    return used


class OBJReader:
    """OBJ file reader.

    load(path)                  -> SceneObject hierarchy
    load_as_mesh(path)          -> flat Mesh made of Triangle objects
    load_as_indexed_mesh(path)  -> flat IndexedMesh backed by shared arrays
    """

    INDEXED_AUTO_THRESHOLD_BYTES = 32 * 1024 * 1024

    @staticmethod
    def load(path, name=None, indexed=None, build_bvh=False, progress=None):
        """Load an OBJ file (obj_reader.py:134-172).  Assimp is not part of
        this package, so non-indexed loads take the Python-structure path."""
        file_path = Path(path)
        if indexed is None:
            indexed = (file_path.suffix.lower() == ".obj"
                       and file_path.stat().st_size >= OBJReader.INDEXED_AUTO_THRESHOLD_BYTES)
        if indexed:
            return OBJReader._load_python_indexed(path, name, build_bvh=build_bvh, progress=progress)
        return OBJReader._load_python(path, name, progress=progress)

    @staticmethod
    def load_as_indexed_mesh(path, build_bvh=False, progress=None):
        """Load an OBJ into IndexedMesh storage without material objects."""
        mesh, _ = OBJReader._parse_indexed(path, build_bvh=build_bvh, progress=progress)
        return mesh

    @staticmethod
    def _parse_indexed(path, build_bvh=False, progress=None):
        """(IndexedMesh, {group: Material}) (obj_reader.py:345-441)."""
        file_path = Path(path)
        tracker = _Progress(progress)
        tracker.emit("Parsing OBJ", str(file_path))
        d = parse_obj(file_path)
        mtl_materials = {}
        for key, parts, _ in d.events:
            if key == "mtllib":
                mtl_materials.update(_load_mtllib(file_path, parts, tracker) or {})
        tracker.track(d)
        tracker.emit("Parsed OBJ", tracker.detail(d))
        tracker.emit("Assembling indexed mesh", tracker.detail(d))
        mesh = IndexedMesh(
            d.positions, d.tri_pos_idx,
            normals=d.normals if len(d.normals) else None, tri_normal_idx=d.tri_normal_idx,
            uvs=d.uvs if len(d.uvs) else None, tri_uv_idx=d.tri_uv_idx,
            groups=d.group_names or ["default"], tri_group_idx=d.tri_group_idx,
            name=file_path.stem, build_bvh=build_bvh)
        used = _tri_ranges_used(d)
        mat_groups = {g: mtl_materials.get(g, _default_material()) for g in (used or {"default"})}
        return mesh, mat_groups

    @staticmethod
    def _load_python_indexed(path, name=None, build_bvh=False, progress=None):
        """SceneObject hierarchy with IndexedMesh leaves (obj_reader.py:174-336):
        `o` and `g` become nodes, runs of one material become leaves."""
        from scene.scene_object import SceneObject
        from scene.shape import Shape as ShapeNode

        file_path = Path(path)
        tracker = _Progress(progress)
        tracker.emit("Parsing OBJ", str(file_path))
        d = parse_obj(file_path)
        root = SceneObject(name=name or file_path.stem)
        mtl_materials = {}
        current_obj_node = current_group_node = root
        current_mtl = "default"
        leaves = []
        pending = [0, "default"]  # first pending triangle, its material name

        def flush(upto):
            if upto > pending[0]:
                leaves.append((current_group_node, current_mtl, pending[0], upto))
            pending[0] = upto

        for key, parts, pre in d.events:
            t = int(pre[_PTRI])
            if key == "mtllib":
                mtl_materials.update(_load_mtllib(file_path, parts, tracker) or {})
            elif key == "o":
                flush(t)
                current_obj_node = SceneObject(name=parts[1] if len(parts) > 1 else "object")
                root.add_child(current_obj_node)
                current_group_node = current_obj_node
            elif key == "g":
                flush(t)
                current_group_node = SceneObject(name=parts[1] if len(parts) > 1 else "group")
                current_obj_node.add_child(current_group_node)
            elif key == "usemtl":
                new_mtl = parts[1] if len(parts) > 1 else "default"
                if new_mtl != current_mtl:
                    flush(t)
                current_mtl = new_mtl
        flush(d.triangle_count)
        tracker.track(d)
        tracker.emit("Parsed OBJ", tracker.detail(d))

        normals = d.normals if len(d.normals) else None
        uvs = d.uvs if len(d.uvs) else None
        for i, (parent, mtl, a, b) in enumerate(leaves, 1):
            tracker.emit("Assembling OBJ meshes", f"{i:,}/{len(leaves):,} mesh leaves • {b - a:,} triangles in current leaf")
            mesh = IndexedMesh(
                d.positions, d.tri_pos_idx[a:b],
                normals=normals, tri_normal_idx=d.tri_normal_idx[a:b],
                uvs=uvs, tri_uv_idx=d.tri_uv_idx[a:b],
                groups=d.group_names or ["default"], tri_group_idx=d.tri_group_idx[a:b],
                name=mtl, build_bvh=build_bvh)
            shape = ShapeNode(mesh, {mtl: mtl_materials.get(mtl, _default_material())}, name=mtl)
            parent.add_child(SceneObject(shapes=[shape], name=mtl))
        tracker.emit("Finished OBJ hierarchy", f"{len(leaves):,} mesh leaves")
        return root

    @staticmethod
    def _triangles(d, a, b, group=None):
        """Triangle objects for rows [a, b) (obj_reader.py:572-583)."""
        if not hasattr(d, "_vecs"):
            d._vecs = ([Vec3(*map(float, p)) for p in d.positions], [Vec3(*map(float, p)) for p in d.normals],
                       [Vec2(*map(float, p)) for p in d.uvs])
        V, N, U = d._vecs
        tris = []
        for t in range(a, b):
            vi, ni, ui = d.tri_pos_idx[t], d.tri_normal_idx[t], d.tri_uv_idx[t]
            kw = {} if group is None else {"group": group}
            tris.append(Triangle(V[vi[0]], V[vi[1]], V[vi[2]],
                                 N[ni[0]] if ni[0] >= 0 else None, N[ni[1]] if ni[1] >= 0 else None,
                                 N[ni[2]] if ni[2] >= 0 else None,
                                 U[ui[0]] if ui[0] >= 0 else None, U[ui[1]] if ui[1] >= 0 else None,
                                 U[ui[2]] if ui[2] >= 0 else None, **kw))
        return tris

    @staticmethod
    def _load_python(path, name=None, progress=None):
        """SceneObject hierarchy with Mesh leaves (obj_reader.py:487-592):
        leaves end at `o` and at a usemtl that changes the material."""
        from scene.scene_object import SceneObject
        from scene.shape import Shape as ShapeNode

        file_path = Path(path)
        tracker = _Progress(progress)
        tracker.emit("Parsing OBJ", str(file_path))
        d = parse_obj(file_path)
        root = SceneObject(name=name or file_path.stem)
        mtl_materials = {}
        current_obj_node = root
        current_mtl = "default"
        start = [0]

        def flush(upto):
            if upto <= start[0]:
                return
            tris = OBJReader._triangles(d, start[0], upto, current_mtl)
            node_name = tris[0].group
            shape = ShapeNode(Mesh(tris), {node_name: mtl_materials.get(node_name, _default_material())},
                              name=node_name)
            current_obj_node.add_child(SceneObject(shapes=[shape], name=node_name))
            start[0] = upto

        for key, parts, pre in d.events:
            t = int(pre[_PTRI])
            if key == "mtllib":
                loaded = _load_mtllib(file_path, parts, tracker)
                if loaded is not None:
                    mtl_materials = loaded
            elif key == "o":
                flush(t)
                current_obj_node = SceneObject(name=parts[1] if len(parts) > 1 else "object")
                root.add_child(current_obj_node)
            elif key == "usemtl":
                new_mtl = parts[1] if len(parts) > 1 else "default"
                if new_mtl != current_mtl and t > start[0]:
                    flush(t)
                current_mtl = new_mtl
        flush(d.triangle_count)
        tracker.track(d)
        tracker.emit("Loaded OBJ", tracker.detail(d))
        return root

    @staticmethod
    def load_as_mesh(path) -> Mesh:
        """One flat Mesh of all triangles, no materials (obj_reader.py:612-646)."""
        d = parse_obj(path)
        return Mesh(OBJReader._triangles(d, 0, d.triangle_count))


__all__ = ["OBJReader", "ObjData", "parse_obj", "parse_obj_bytes"]
