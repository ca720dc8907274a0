"""Scene file formats on the host: RXB archives (scene/io/roxy_binary.py)
and MTL libraries (scene/io/mtl_loader.py).  No GPU needed."""
import os

import numpy as np
import pytest

from scene.io.mtl_loader import MTLLoader
from scene.io.roxy_binary import (list_rxb_meshes, load_rxb_mesh, load_rxb_mesh_ref, load_rxb_metadata,
                                  save_rxb_meshes, split_rxb_mesh_ref)
from scene.materials import Dielectric, Diffuse, Emissive, Glossy, Metal
from scene.mesh import IndexedMesh

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _golden_meshes():
    """The meshes tests/golden/make_golden.py (make_rxb) gave the reference's
    save_rxb_meshes, rebuilt from the same seed."""
    rng = np.random.default_rng(11)
    pos = rng.normal(size=(40, 3))
    a = dict(positions=pos, tri_pos_idx=rng.integers(0, 40, size=(25, 3)), normals=rng.normal(size=(40, 3)),
             tri_normal_idx=rng.integers(0, 40, size=(25, 3)), uvs=rng.random((40, 2)),
             tri_uv_idx=rng.integers(0, 40, size=(25, 3)), groups=["paint", "rubber"],
             tri_group_idx=rng.integers(0, 2, size=25), name="frame")
    b = dict(positions=pos, tri_pos_idx=rng.integers(0, 40, size=(7, 3)), name="wheel")
    return a, b


def _same(mesh, want):
    np.testing.assert_array_equal(mesh._positions, want["positions"])
    np.testing.assert_array_equal(mesh._tri_pos_idx, want["tri_pos_idx"])
    if "normals" in want:
        np.testing.assert_array_equal(mesh._normals, want["normals"])
        np.testing.assert_array_equal(mesh._tri_normal_idx, want["tri_normal_idx"])
        np.testing.assert_array_equal(mesh._uvs, want["uvs"])
        np.testing.assert_array_equal(mesh._tri_uv_idx, want["tri_uv_idx"])
        np.testing.assert_array_equal(mesh._tri_group_idx, want["tri_group_idx"])
        assert mesh.groups == want["groups"]
    else:
        assert mesh._normals is None and mesh._uvs is None
        assert (mesh._tri_normal_idx == -1).all() and (mesh._tri_uv_idx == -1).all()
    assert mesh._name == want["name"]


def test_reads_an_archive_the_reference_wrote():
    path = os.path.join(GOLD, "meshes.rxb")
    a, b = _golden_meshes()
    assert list_rxb_meshes(path) == ["frame", "parts/wheel"]
    meta = load_rxb_metadata(path)
    assert meta["format"] == "rxb" and meta["version"] == 2
    # one shared positions buffer
    assert meta["meshes"]["frame"]["positions_buffer"] == meta["meshes"]["parts/wheel"]["positions_buffer"]
    cache = {}
    fa = load_rxb_mesh(path, "frame", cache=cache)
    fb = load_rxb_mesh_ref("meshes.rxb:meshes/parts/wheel", base_dir=GOLD, cache=cache)
    _same(fa, a)
    _same(fb, b)
    assert np.shares_memory(fa._positions, fb._positions)  # shared through the cache


def test_written_archive_matches_the_reference_layout(tmp_path):
    a, b = _golden_meshes()
    ma = IndexedMesh(**{k: v for k, v in a.items()})
    mb = IndexedMesh(ma._positions, b["tri_pos_idx"], name="wheel")
    out = tmp_path / "out.rxb"
    save_rxb_meshes(out, {"frame": ma, "parts/wheel": mb})
    ref = np.load(os.path.join(GOLD, "meshes.rxb"))
    mine = np.load(out)
    assert sorted(ref.files) == sorted(mine.files)
    for k in ref.files:
        assert ref[k].dtype == mine[k].dtype and ref[k].shape == mine[k].shape, k
        np.testing.assert_array_equal(ref[k], mine[k], err_msg=k)
    _same(load_rxb_mesh(out, "frame"), a)


def test_rxb_errors(tmp_path):
    path = os.path.join(GOLD, "meshes.rxb")
    with pytest.raises(KeyError, match="available: frame, parts/wheel"):
        load_rxb_mesh(path, "nope")
    with pytest.raises(ValueError):
        split_rxb_mesh_ref("no_colon_here")
    with pytest.raises(ValueError):
        split_rxb_mesh_ref("file.rxb:meshes/")
    assert split_rxb_mesh_ref("a/b.rxb:x", base_dir="/base") == (__import__("pathlib").Path("/base/a/b.rxb"), "x")
    with pytest.raises(TypeError):
        save_rxb_meshes(tmp_path / "bad.rxb", {"x": object()})
    bad = tmp_path / "bad.rxb"
    with open(bad, "wb") as f:
        np.savez(f, __metadata__=np.frombuffer(b'{"format":"other","meshes":{}}', np.uint8))
    with pytest.raises(ValueError, match="not a Roxy Binary"):
        load_rxb_mesh(bad, "x")


def test_mtl_loader_maps_materials(tmp_path):
    p = tmp_path / "m.mtl"
    p.write_text("# comment\n"
                 "newmtl light\nKe 4 4 4\n"
                 "newmtl glass\nd 0.5\nNi 1.45\nTf 0.9 1 1\n"
                 "newmtl chrome\nillum 3\nKd 0.8 0.8 0.8\nNs 250\n"
                 "newmtl shiny\nKd 0.2 0.3 0.4\nKs 1 1 1 # trailing\nNs 500\n"
                 "newmtl plain\nKd 0.5 0.25 0.125\nmap_Kd textures/wood.png\n"
                 "newmtl seethru\nTr 0.3\n")
    mats = MTLLoader.load(str(p))
    assert list(mats) == ["light", "glass", "chrome", "shiny", "plain", "seethru"]
    assert isinstance(mats["light"].to_material(), Emissive)
    g = mats["glass"].to_material()
    assert isinstance(g, Dielectric) and abs(g._ior - 1.45) < 1e-12
    m = mats["chrome"].to_material()
    assert isinstance(m, Metal) and abs(m._roughness - 0.75) < 1e-12
    s = mats["shiny"].to_material()
    assert isinstance(s, Glossy) and abs(s._roughness - 0.5) < 1e-12
    d = mats["plain"].to_material()
    assert isinstance(d, Diffuse) and d._albedo_texture is not None
    assert mats["plain"].map_kd == str(tmp_path / "textures" / "wood.png")
    assert abs(mats["seethru"].d - 0.7) < 1e-12 and isinstance(mats["seethru"].to_material(), Dielectric)
