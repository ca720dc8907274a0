"""Roxy Binary (RXB) mesh archives (scene/io/roxy_binary.py:13-237).

An RXB file is an uncompressed NumPy .npz archive: one JSON metadata member
("__metadata__", UTF-8 bytes as uint8) and plain arrays.  Vertex buffers
(float64 positions / normals / uvs) are stored once per distinct array and
shared by the meshes that use them ("buffer.<kind>_<n>"); each mesh adds its
int32 index tables ("mesh_<i>.tri_pos_idx", ".tri_normal_idx",
".tri_uv_idx", ".tri_group_idx").  Files written here load in the
reference and the other way round: the member names, dtypes and metadata
keys are the format.
"""
import json
from pathlib import Path

import numpy as np

from scene.mesh import IndexedMesh

RXB_FORMAT_VERSION = 2
_METADATA_KEY = "__metadata__"
_TABLES = ("tri_pos_idx", "tri_normal_idx", "tri_uv_idx", "tri_group_idx")


def _array_identity(a):
    """Arrays that are the same memory view share one stored buffer."""
    return (a.__array_interface__["data"][0], a.shape, str(a.dtype), a.strides)


def save_rxb_meshes(path, meshes):
    """Write {name: IndexedMesh} (or (name, mesh) pairs) to an RXB file."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    items = list(meshes.items()) if hasattr(meshes, "items") else list(meshes)
    meta = {"format": "rxb", "version": RXB_FORMAT_VERSION, "buffers": {}, "meshes": {}}
    arrays, seen = {}, {}
    per_kind = {"positions": 0, "normals": 0, "uvs": 0}

    def store(kind, value):
        if value is None:
            return None
        a = np.asarray(value, dtype=np.float64)
        key = (kind, _array_identity(a))
        if key not in seen:
            buffer_id = f"{kind}_{per_kind[kind]}"
            per_kind[kind] += 1
            arrays[f"buffer.{buffer_id}"] = a
            meta["buffers"][buffer_id] = {"kind": kind, "array": f"buffer.{buffer_id}", "dtype": str(a.dtype),
                                          "shape": list(a.shape)}
            seen[key] = buffer_id
        return seen[key]

    for i, (name, mesh) in enumerate(items):
        if not isinstance(mesh, IndexedMesh):
            raise TypeError(f"RXB mesh payload {name!r} is not an IndexedMesh")
        prefix = f"mesh_{i}"
        meta["meshes"][name] = {
            "prefix": prefix,
            "name": mesh._name,
            "groups": list(mesh._groups),
            "has_normals": mesh._normals is not None,
            "has_uvs": mesh._uvs is not None,
            "positions_buffer": store("positions", mesh._positions),
            "normals_buffer": store("normals", mesh._normals),
            "uvs_buffer": store("uvs", mesh._uvs),
            "vertex_count": mesh.vertex_count,
            "triangle_count": mesh.triangle_count,
        }
        for t in _TABLES:
            arrays[f"{prefix}.{t}"] = np.asarray(getattr(mesh, "_" + t), dtype=np.int32)
    encoded = json.dumps(meta, separators=(",", ":"), sort_keys=True).encode("utf-8")
    arrays[_METADATA_KEY] = np.frombuffer(encoded, dtype=np.uint8)
    with open(path, "wb") as f:
        np.savez(f, **arrays)


def _read_metadata(archive):
    return json.loads(bytes(np.asarray(archive[_METADATA_KEY], dtype=np.uint8)).decode("utf-8"))


def _check(meta, path):
    if meta.get("format") != "rxb":
        raise ValueError(f"{path} is not a Roxy Binary file")
    if meta.get("version") not in (1, RXB_FORMAT_VERSION):
        raise ValueError(f"Unsupported RXB version {meta.get('version')} in {path}; expected {RXB_FORMAT_VERSION}")


def load_rxb_metadata(path):
    with np.load(path, allow_pickle=False) as archive:
        return _read_metadata(archive)


def list_rxb_meshes(path):
    return list(load_rxb_metadata(path).get("meshes", {}).keys())


def _buffer(path, archive, meta, buffer_id, cache):
    info = meta.get("buffers", {}).get(buffer_id)
    if info is None:
        raise KeyError(f"RXB buffer {buffer_id!r} not found in {path}")
    key = (str(Path(path).resolve()), buffer_id)
    if cache is not None and key in cache:
        return cache[key]
    a = np.array(archive[info["array"]], copy=True)
    if cache is not None:
        cache[key] = a
    return a


def _vertex_array(path, archive, meta, m, prefix, legacy, cache, optional=True):
    """A mesh's vertex buffer: shared (version 2) or per mesh (version 1)."""
    if optional and not m.get(f"has_{legacy}"):
        return None
    buffer_id = m.get(f"{legacy}_buffer")
    if buffer_id:
        return _buffer(path, archive, meta, buffer_id, cache)
    return np.array(archive[f"{prefix}.{legacy}"], copy=True)


def load_rxb_mesh(path, name, build_bvh=False, cache=None):
    """IndexedMesh `name` of an RXB file; `cache` (a dict) shares vertex
    buffers between loads of meshes from the same file."""
    path = Path(path)
    with np.load(path, allow_pickle=False) as archive:
        meta = _read_metadata(archive)
        _check(meta, path)
        try:
            m = meta["meshes"][name]
        except KeyError as exc:
            available = ", ".join(meta["meshes"].keys())
            raise KeyError(f"RXB mesh {name!r} not found in {path}; available: {available}") from exc
        prefix = m["prefix"]
        tables = {t: np.array(archive[f"{prefix}.{t}"], copy=True) for t in _TABLES}
        return IndexedMesh(
            _vertex_array(path, archive, meta, m, prefix, "positions", cache, optional=False),
            tables["tri_pos_idx"],
            normals=_vertex_array(path, archive, meta, m, prefix, "normals", cache),
            tri_normal_idx=tables["tri_normal_idx"],
            uvs=_vertex_array(path, archive, meta, m, prefix, "uvs", cache),
            tri_uv_idx=tables["tri_uv_idx"],
            groups=m.get("groups") or ["default"],
            tri_group_idx=tables["tri_group_idx"],
            name=m.get("name", name),
            build_bvh=build_bvh,
        )


def split_rxb_mesh_ref(ref, base_dir=None):
    """'file.rxb:meshes/name' (or 'file.rxb:name') -> (path, name)."""
    if ":" not in ref:
        raise ValueError(f"RXB mesh references must look like file.rxb:meshes/name: {ref}")
    path_text, mesh_path = ref.rsplit(":", 1)
    name = mesh_path[len("meshes/"):] if mesh_path.startswith("meshes/") else mesh_path
    if not name:
        raise ValueError(f"RXB mesh reference is missing a mesh name: {ref}")
    path = Path(path_text)
    if not path.is_absolute() and base_dir is not None:
        path = Path(base_dir) / path
    return path, name


def load_rxb_mesh_ref(ref, base_dir=None, build_bvh=False, cache=None):
    path, name = split_rxb_mesh_ref(ref, base_dir=base_dir)
    return load_rxb_mesh(path, name, build_bvh=build_bvh, cache=cache)


__all__ = ["RXB_FORMAT_VERSION", "save_rxb_meshes", "load_rxb_metadata", "list_rxb_meshes", "load_rxb_mesh",
           "load_rxb_mesh_ref", "split_rxb_mesh_ref"]
