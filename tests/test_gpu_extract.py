"""Scene extraction on the device (rx_scene_put_indexed / put_triangles):
the float32 rows it writes equal the reference's
IndexedMesh.indexed_triangle_arrays (golden vectors) and, for whole worlds,
the host flattening of collect() + GPUBVHBuilder (triangles, palette
indices, palette and light list), bit for bit."""
import os

import numpy as np
import pytest

import golden_scenes as gs
import roxy_native as nat
import workloads
from rendering.taichi.extractor import HostScene, build_device_scene
from rendering.taichi.lights import build_lights
from test_host_logic import _ns

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROWS = ("v0", "v1", "v2", "n0", "n1", "n2")


def _bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _put_object(sc, offset, obj, group_mat):
    geo = obj.shapes[0].geometry
    sc.put_indexed(offset, geo._positions, geo._tri_pos_idx, geo._normals, geo._tri_normal_idx,
                   obj.world_matrix.rows, obj.world_inverse_transpose_matrix.rows, geo._tri_group_idx, group_mat)
    return geo.triangle_count


def test_put_indexed_matches_reference_golden():
    g = np.load(os.path.join(GOLD, "indexed_arrays.npz"))
    obj = gs.build_indexed_object(_ns())
    sc = nat.NativeScene()
    n = obj.shapes[0].geometry.triangle_count
    sc.alloc_triangles(n)
    _put_object(sc, 0, obj, [5, 9])
    got = sc.get_triangles()
    for k in ROWS:
        assert _bits_equal(got[k], g[k]), k
    np.testing.assert_array_equal(got["mat_idx"], np.where(g["group_idx"] == 1, 9, 5))


def test_put_pieces_at_offsets():
    """Two indexed pieces and a row piece land at their offsets; unwritten
    rows stay zero."""
    g = np.load(os.path.join(GOLD, "indexed_arrays.npz"))
    obj = gs.build_indexed_object(_ns())
    n = obj.shapes[0].geometry.triangle_count
    v0, v1, v2 = gs.soup_triangles(37, 3)
    sc = nat.NativeScene()
    sc.alloc_triangles(2 * n + 37 + 5)
    _put_object(sc, 0, obj, [1, 2])
    sc.put_triangles(n, v0, v1, v2, v0, v1, v2, np.full(37, 7, np.int32))
    _put_object(sc, n + 37, obj, [3, 4])
    got = sc.get_triangles()
    for k in ROWS:
        assert _bits_equal(got[k][:n], g[k]), k
        assert _bits_equal(got[k][n + 37:2 * n + 37], g[k]), k
        assert not got[k][2 * n + 37:].any()
    assert _bits_equal(got["v1"][n:n + 37], v1) and _bits_equal(got["n2"][n:n + 37], v2)
    np.testing.assert_array_equal(got["mat_idx"][n:n + 37], 7)
    np.testing.assert_array_equal(got["mat_idx"][2 * n + 37:], 0)


def test_large_row_arrays_round_trip_through_the_pinned_stage():
    """Arrays of several MB go through the context's pinned buffer in 2 MB
    pieces (host copies on worker threads, one DMA per piece), both ways;
    lengths that end inside a piece and an offset that is not piece aligned
    come back bit for bit, and the rows around them stay zero."""
    rng = np.random.default_rng(7)
    n = 600_017  # 7.2 MB per row array: three full pieces and a partial one
    rows = [rng.standard_normal((n, 3)).astype(np.float32) for _ in range(6)]
    mat = rng.integers(0, 1000, n).astype(np.int32)
    sc = nat.NativeScene()
    sc.alloc_triangles(n + 12)
    sc.put_triangles(5, *rows, mat)
    got = sc.get_triangles()
    for k, r in zip(ROWS, rows):
        assert _bits_equal(got[k][5:5 + n], r), k
        assert not got[k][:5].any() and not got[k][5 + n:].any(), k
    np.testing.assert_array_equal(got["mat_idx"][5:5 + n], mat)
    np.testing.assert_array_equal(got["mat_idx"][:5], 0)
    # a second upload over part of the rows reuses the buffer
    sc.put_triangles(100, rows[1][:300_000], rows[2][:300_000], rows[0][:300_000])
    got = sc.get_triangles(100, 300_000)
    assert _bits_equal(got["v0"], rows[1][:300_000]) and _bits_equal(got["v2"], rows[0][:300_000])
    assert _bits_equal(got["n1"], rows[1][:300_000])  # absent normal rows repeat v0


def test_put_indexed_rejects_bad_indices():
    sc = nat.NativeScene()
    pos = np.eye(3)
    sc.alloc_triangles(2)
    with pytest.raises(ValueError, match="position index"):
        sc.put_indexed(0, pos, [[0, 1, 2], [0, 1, 3]], group_mat=[0])
    with pytest.raises(ValueError, match="normal index"):
        sc.put_indexed(0, pos, [[0, 1, 2], [0, 1, 2]], normals=pos, tri_normal_idx=[[0, 1, 2], [0, 4, 1]],
                       group_mat=[0])
    with pytest.raises(ValueError, match="group index"):
        sc.put_indexed(0, pos, [[0, 1, 2], [0, 1, 2]], tri_group_idx=[0, 2], group_mat=[0, 1])
    with pytest.raises(ValueError, match="outside"):
        sc.put_indexed(1, pos, [[0, 1, 2], [0, 1, 2]], group_mat=[0])
    with pytest.raises(ValueError, match="outside"):
        sc.put_triangles(2, pos[:1], pos[:1], pos[:1])
    # the scene is still usable after the rejected calls
    sc.put_indexed(0, pos, [[0, 1, 2], [2, 1, 0]], group_mat=[0])
    got = sc.get_triangles()
    assert _bits_equal(got["v0"], [[1, 0, 0], [0, 0, 1]])


def _mixed_world():
    ns = _ns()
    world = gs.build_trace_scene(ns)
    world.add_object(gs.build_indexed_object(ns))
    return world


@pytest.mark.parametrize("name", ["trace", "mixed", "cornell", "icosphere", "icosphere_full", "texture",
                                  "texture_indexed"])
def test_device_extraction_equals_host_flattening(name):
    # icosphere_full: the 327,680-triangle mesh of the benchmark, whose 17 MB
    # of index and position arrays go through the staged upload in pieces
    world = {"trace": lambda: gs.build_trace_scene(_ns()), "mixed": _mixed_world,
             "cornell": lambda: workloads.cornell_box(64, 64),
             "icosphere": lambda: workloads.displaced_icosphere_scene(64, 36, subdiv=4),
             "icosphere_full": lambda: workloads.displaced_icosphere_scene(64, 36),
             "texture": lambda: gs.build_texture_scene(_ns()),
             "texture_indexed": lambda: gs.build_texture_scene(_ns(), indexed=True)}[name]()
    ds = build_device_scene(world, method="lbvh")
    h = HostScene(world)
    got = ds.native.get_triangles()
    b = h.batch
    for k in ROWS:
        assert _bits_equal(got[k], getattr(b, k)), k
    np.testing.assert_array_equal(got["mat_idx"], h.mat_idx)
    pal = ds._light_args[4:]
    np.testing.assert_array_equal(pal[0], h.palette[0])
    assert _bits_equal(pal[1], h.palette[1]) and _bits_equal(pal[2], h.palette[4])
    np.testing.assert_array_equal(ds.pal_texture, h.mat_texture)
    assert ds.stats["bvh_triangles"] == b.triangle_count
    assert ds.stats["bvh_materials"] == len(h.builder.mat_palette)
    for compat in (False, True):
        a = build_lights(ds.slots, *ds._light_args, compat=compat, pal_texture=ds.pal_texture,
                         tri_index=ds._light_index)
        r = h.lights(compat)
        assert (a is None) == (r is None)
        if a is not None:
            for k in r:
                np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(r[k]), err_msg=f"{name}:{k}")
