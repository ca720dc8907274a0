"""Device OBJ parser (rx_obj_* behind scene.io.obj_reader.OBJReader) against
the reference's reader (golden fixtures written by running
scene/io/obj_reader.py on the same text) and the CPU restatement
(oracle.obj_parse) on larger seeded texts."""
import json
import os

import numpy as np
import pytest

from make_golden import _obj_text
from oracle.obj_parse import parse_indexed
from scene.io.obj_reader import OBJReader, parse_obj_bytes
from scene.mesh import IndexedMesh, Mesh

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ARRAYS = ("positions", "normals", "uvs", "tri_pos_idx", "tri_normal_idx", "tri_uv_idx", "tri_group_idx")


def _bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype == np.float64 or b.dtype == np.float64:
        a, b = a.astype(np.float64), b.astype(np.float64)
        return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
    return a.shape == b.shape and np.array_equal(a, b)


def _tree(node, indexed):
    shapes = [{"name": s.name, "groups": sorted(s.material_groups.keys()),
               "tris": int(s.geometry.triangle_count if indexed else len(s.geometry._triangles))}
              for s in node.shapes]
    return {"name": node.name, "shapes": shapes, "children": [_tree(c, indexed) for c in node.children]}


@pytest.mark.parametrize("name", ["obj_small", "obj_random"])
def test_device_parse_matches_reference_reader(name, tmp_path, capsys):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    meta = json.loads(bytes(g["meta"]).decode())
    path = tmp_path / (name + ".obj")
    path.write_bytes(bytes(g["text"]))
    mesh, mat_groups = OBJReader._parse_indexed(path)
    assert (mesh._normals is not None) == bool(g["has_normals"])
    assert (mesh._uvs is not None) == bool(g["has_uvs"])
    got = {"positions": mesh._positions, "normals": mesh._normals if mesh._normals is not None else np.zeros((0, 3)),
           "uvs": mesh._uvs if mesh._uvs is not None else np.zeros((0, 2)), "tri_pos_idx": mesh._tri_pos_idx,
           "tri_normal_idx": mesh._tri_normal_idx, "tri_uv_idx": mesh._tri_uv_idx,
           "tri_group_idx": mesh._tri_group_idx}
    for k in ARRAYS:
        assert _bits_equal(got[k], g[k]), k
    assert mesh.groups == meta["groups"]
    assert sorted(mat_groups) == meta["mat_groups"]
    assert capsys.readouterr().out.splitlines() == meta["warnings"]
    assert _tree(OBJReader.load(path, indexed=True), True) == meta["tree_indexed"]
    assert _tree(OBJReader.load(path, indexed=False), False) == meta["tree_python"]


@pytest.mark.parametrize("seed,blocks", [(3, 20000), (5, 3000)])
def test_device_parse_matches_restatement_on_large_text(seed, blocks):
    text = _obj_text(seed, blocks).encode("utf-8")
    d = parse_obj_bytes(text)
    r = parse_indexed(text)
    for k in ARRAYS:
        assert _bits_equal(getattr(d, k), r[k]), k
    assert d.group_names == r["groups"]
    assert d.triangle_count > 10 * blocks // 4


def test_line_endings_whitespace_and_empty_texts():
    assert parse_obj_bytes(b"").triangle_count == 0
    assert parse_obj_bytes(b"# only a comment").positions.shape == (0, 3)
    for text in (b"v 0 0 0\rv 1 0 0\rv 0 1 0\rf 1 2 3",          # lone CR, no final newline
                 b"v 0 0 0\r\nv 1 0 0\r\nv 0 1 0\r\nf 1 2 3\r\n",  # CRLF
                 b"\tv\t0 0 0\x0b\nv 1\x0c0 0\n v 0 1 0 \nf\x1c1 2 3\n"):  # str.split() whitespace
        d = parse_obj_bytes(text)
        r = parse_indexed(text)
        for k in ARRAYS:
            assert _bits_equal(getattr(d, k), r[k]), (text, k)
        assert d.triangle_count == 1


def test_numbers_the_device_does_not_convert_go_through_float():
    text = (b"v 1_000.5 -0.0 1e-400\nv 12345678901234567890.5 nan -inf\n"
            b"v 0.30000000000000004 9007199254740993 1e23\nf 1 2 3\n")
    d = parse_obj_bytes(text)
    r = parse_indexed(text)
    assert _bits_equal(d.positions, r["positions"])
    assert np.signbit(d.positions[0, 1]) and np.isnan(d.positions[1, 1])


def test_errors_match_the_reference():
    with pytest.raises(IndexError):
        parse_obj_bytes(b"v 1 2\n")
    with pytest.raises(ValueError):
        parse_obj_bytes(b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 a 3\n")
    with pytest.raises(ValueError):
        parse_obj_bytes(b"v 0 0 0\nf /1 1 1\n")
    with pytest.raises(UnicodeDecodeError):
        parse_obj_bytes(b"v 0 0 0\n# \xff\xfe\n")


def test_non_ascii_lines_are_split_as_python_splits_them():
    # U+00A0 is whitespace to str.split(): "v\xa01 2 3" is a vertex line
    text = "v 1 2 3\nv 4 5 6 \nv 7 8 9\nusemtl métal\nf 1 2 3\n".encode("utf-8")
    d = parse_obj_bytes(text)
    r = parse_indexed(text)
    for k in ARRAYS:
        assert _bits_equal(getattr(d, k), r[k]), k
    assert d.group_names == ["default", "métal"]


def _write(tmp_path, text):
    p = tmp_path / "m.obj"
    p.write_text(text)
    return p


def test_reference_reader_contracts(tmp_path):
    """The reference's obj_reader_tests cases that need the parse."""
    p = _write(tmp_path, "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    assert len(OBJReader.load_as_mesh(p)._triangles) == 2
    p = _write(tmp_path, "v 1 0 0\nv 0.309 0.951 0\nv -0.809 0.588 0\nv -0.809 -0.588 0\nv 0.309 -0.951 0\n"
                         "f 1 2 3 4 5\n")
    assert len(OBJReader.load_as_mesh(p)._triangles) == 3
    p = _write(tmp_path, "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvn 0 0 1\nvn 0 0 1\nvn 0 0 1\n"
                         "f 1/1/1 2/2/2 3/3/3\n")
    tri = OBJReader.load_as_mesh(p)._triangles[0]
    assert tri._uv0 is not None and tri._n0 is not None and tri._uv1[0] == 1.0
    p = _write(tmp_path, "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    assert OBJReader.load_as_mesh(p)._triangles[0]._n0 is None
    m = OBJReader.load_as_indexed_mesh(p)
    assert isinstance(m, IndexedMesh) and m.vertex_count == 3 and m.triangle_count == 1
    root = OBJReader.load(p)
    assert isinstance(root.children[0].shapes[0].geometry, Mesh)
    p = _write(tmp_path, "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nv 1 0 1\nv 0 1 1\n"
                         "usemtl matA\nf 1 2 3\nusemtl matB\nf 4 5 6\n")
    m = OBJReader.load_as_indexed_mesh(p)
    assert m.groups == ["default", "matA", "matB"]
    assert m.group_for_triangle(0) == "matA" and m.group_for_triangle(1) == "matB"
    assert [c.name for c in OBJReader.load(p).children] == ["matA", "matB"]
    root = OBJReader.load(p, indexed=True)
    assert [set(c.shapes[0].material_groups) for c in root.children] == [{"matA"}, {"matB"}]
    p = _write(tmp_path, "o BikeFrame\ng FrontTriangle\nv 0 0 0\nv 1 0 0\nv 0 1 0\nusemtl matA\nf 1 2 3\n"
                         "g RearTriangle\nv 0 0 1\nv 1 0 1\nv 0 1 1\nusemtl matB\nf 4 5 6\n")
    events = []
    root = OBJReader.load(p, indexed=True, progress=lambda t, d: events.append((t, d)))
    obj = root.children[0]
    assert obj.name == "BikeFrame" and [c.name for c in obj.children] == ["FrontTriangle", "RearTriangle"]
    assert obj.children[0].children[0].name == "matA" and obj.children[1].children[0].name == "matB"
    assert any(t == "Parsed OBJ" for t, _ in events)
    assert any("2 tris" in d for _, d in events) and any("object: BikeFrame" in d for _, d in events)


def test_materials_from_mtllib(tmp_path):
    (tmp_path / "lib.mtl").write_text("newmtl glow\nKe 1 2 3\nnewmtl base\nKd 0.1 0.2 0.3\n")
    p = _write(tmp_path, "mtllib lib.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nusemtl glow\nf 1 2 3\nusemtl base\nf 3 2 1\n"
                         "usemtl unused\n")
    _, mats = OBJReader._parse_indexed(p)
    assert sorted(mats) == ["base", "glow"]
    assert type(mats["glow"]).__name__ == "Emissive" and type(mats["base"]).__name__ == "Diffuse"
