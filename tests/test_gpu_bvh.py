"""GPU BVH builds: the reference Morton build is bit-exact against the
reference builder's golden output and the oracle; the LBVH satisfies the
structural invariants (every primitive in exactly one leaf, every box
contains its primitives)."""
import os

import numpy as np
import pytest

import golden_scenes as gs
import roxy_native as nat
from oracle import oracle
from rendering.taichi.bvh_builder import GPUBVHBuilder, TriangleBatch

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _batch(v0, v1, v2):
    n = len(v0)
    z = np.tile(np.float32([0, 0, 1]), (n, 1))
    return TriangleBatch(v0, v1, v2, z, z, z, np.zeros(n, np.int32), np.ones((n, 3), np.float32),
                         np.zeros(n, np.float32), np.ones(n, np.float32), np.zeros(n, np.float32))


def _tri(x, **kw):
    d = {'v0': [x, 0, 0], 'v1': [x + 1, 0, 0], 'v2': [x, 1, 0], 'n0': [0, 0, 1], 'n1': [0, 0, 1], 'n2': [0, 0, 1],
         'mat_type': 0, 'albedo': [1, 1, 1], 'roughness': 0.0, 'ior': 1.0, 'emission': 0.0}
    d.update(kw)
    return d


def _node_arrays(builder):
    nodes = list(builder.nodes)
    return dict(node_min=np.array([n['aabb_min'] for n in nodes], np.float32),
                node_max=np.array([n['aabb_max'] for n in nodes], np.float32),
                left=np.array([n['left'] for n in nodes], np.int32), right=np.array([n['right'] for n in nodes], np.int32),
                start=np.array([n['tri_start'] for n in nodes], np.int32),
                count=np.array([n['tri_count'] for n in nodes], np.int32))


def test_reference_build_bit_exact_against_reference_builder():
    g = np.load(os.path.join(GOLD, "bvh_build.npz"))
    for case in g["case_names"]:
        c = {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith(f"{case}/")}
        b = GPUBVHBuilder()
        b.MAX_LEAF_SIZE = int(c["leaf"])
        b.build([_batch(c["v0"], c["v1"], c["v2"])])
        got = _node_arrays(b)
        for k in ("left", "right", "start", "count"):
            np.testing.assert_array_equal(got[k], c[k], err_msg=f"{case}:{k}")
        for k in ("node_min", "node_max"):
            assert np.array_equal(got[k].view(np.uint32), c[k].view(np.uint32)), f"{case}:{k}"
        np.testing.assert_array_equal(b.ordered_tris, c["order"], err_msg=case)


def test_reference_builder_contracts():
    # the reference's own tests (tests/bvh_builder_tests.py)
    b = GPUBVHBuilder().build([_tri(0), _tri(2)])
    assert b.triangle_count == 2 and len(b.nodes) == 1 and len(b.mat_palette) == 1
    batch = TriangleBatch.from_dicts([_tri(0), _tri(2, albedo=[0.5, 0.5, 0.5])])
    b = GPUBVHBuilder().build([batch])
    assert b.triangle_count == 2 and len(b.nodes) == 1 and len(b.mat_palette) == 2
    assert b._ordered_v0.shape == (2, 3)
    b = GPUBVHBuilder()
    b.MAX_LEAF_SIZE = 4
    b.build([TriangleBatch.from_dicts([_tri(x) for x in range(8)])])
    assert b.triangle_count == 8 and len(b.nodes) == 3
    assert b.nodes[0]['left'] > 0 and b.nodes[0]['right'] > 0
    b = GPUBVHBuilder()
    b.MAX_LEAF_SIZE = 1
    b.build([TriangleBatch.from_dicts([_tri(x) for x in [7, 1, 6, 0, 5, 2, 4, 3]])])
    assert list(b._ordered_v0[:, 0]) == [0, 1, 2, 3, 4, 5, 6, 7]
    b = GPUBVHBuilder()
    b.MAX_LEAF_SIZE = 1
    b.build([TriangleBatch.from_dicts([_tri(x) for x in [7, 1, 6, 0, 5, 2, 4, 3]])], method="median")

    def check(i):
        nd = b.nodes[i]
        if nd['left'] == -1:
            return
        axis = b._longest_axis(nd['aabb_min'], nd['aabb_max'])
        assert b.nodes[nd['left']]['aabb_max'][axis] <= b.nodes[nd['right']]['aabb_max'][axis]
        check(nd['left'])
        check(nd['right'])

    check(0)
    with pytest.raises(ValueError):
        GPUBVHBuilder().build([_tri(0)], method="bogus")


def test_large_reference_build_matches_oracle():
    pos, f = gs.icosphere(6)
    rng = np.random.default_rng(5)
    pos = pos * (1 + 0.05 * rng.standard_normal(len(pos)))[:, None]
    v0, v1, v2 = (pos[f[:, k]].astype(np.float32) for k in range(3))
    b = GPUBVHBuilder().build([_batch(v0, v1, v2)])
    ref = oracle.bvh_build_morton(v0, v1, v2, 8)
    got = _node_arrays(b)
    for k in ("left", "right", "start", "count"):
        np.testing.assert_array_equal(got[k], ref[k])
    assert np.array_equal(got["node_min"].view(np.uint32), ref["node_min"].view(np.uint32))
    np.testing.assert_array_equal(b.ordered_tris, ref["order"])


def _check_layout(nodes, order, n_prims, pmin, pmax):
    """Every primitive reached exactly once; every child box holds its prims."""
    seen = np.zeros(n_prims, np.int32)
    ints = nodes.view(np.int32)
    stack = [0]
    internal = 0
    while stack:
        i = stack.pop()
        internal += 1
        box = nodes[i]
        for side in (0, 1):
            lo = np.array([box[0], box[2], box[4]] if side == 0 else [box[6], box[8], box[10]])
            hi = np.array([box[1], box[3], box[5]] if side == 0 else [box[7], box[9], box[11]])
            w, c = ints[i, 12 + side], ints[i, 14 + side]
            if w >= 0:
                stack.append(w)
                continue
            first, packed_count = (~w) >> 5, (~w) & 31
            assert packed_count == c
            for k in range(first, first + c):
                p = order[k]
                seen[p] += 1
                assert np.all(pmin[p] >= lo - 1e-6) and np.all(pmax[p] <= hi + 1e-6)
    assert internal == len(nodes)
    np.testing.assert_array_equal(seen, 1)


@pytest.mark.parametrize("n,leaf", [(1, 4), (2, 4), (3, 1), (1000, 4), (20000, 4), (20000, 8)])
def test_lbvh_structure(n, leaf):
    v0, v1, v2 = gs.soup_triangles(n, 100 + n)
    sc = nat.NativeScene()
    sc.set_triangles(v0, v1, v2)
    sc.set_materials([0], [[0.5, 0.5, 0.5]], [0.0], [1.0], [0.0])
    sc.build_bvh(nat.RX_BVH_LBVH_SAH, leaf, True)
    nodes, order = sc.export_layout()
    st = np.stack([v0, v1, v2], 1)
    _check_layout(nodes, order, n, st.min(1) - 1e-4, st.max(1) + 1e-4)


def test_lbvh_with_spheres_in_tree():
    v0, v1, v2 = gs.soup_triangles(500, 7)
    sc = nat.NativeScene()
    rng = np.random.default_rng(3)
    k = 40
    slots = dict(type=np.zeros(k, np.int32), center=rng.uniform(-1, 1, (k, 3)), radius=rng.uniform(0.01, 0.1, k),
                 normal=np.zeros((k, 3)), offset=np.zeros(k), extra=np.zeros((k, 3)), v0=np.zeros((k, 3)),
                 v1=np.zeros((k, 3)), v2=np.zeros((k, 3)), mat_type=np.zeros(k, np.int32), albedo=np.ones((k, 3)),
                 roughness=np.zeros(k), ior=np.ones(k), emission=np.zeros(k))
    sc.set_objects(slots)
    sc.set_triangles(v0, v1, v2)
    sc.set_materials([0], [[0.5, 0.5, 0.5]], [0.0], [1.0], [0.0])
    sc.build_bvh(nat.RX_BVH_LBVH_SAH, 4, True)
    nodes, order = sc.export_layout()
    st = np.stack([v0, v1, v2], 1)
    c = slots["center"].astype(np.float32)
    r = slots["radius"].astype(np.float32)[:, None]
    pmin = np.concatenate([st.min(1) - 1e-4, c - r - 1e-4])
    pmax = np.concatenate([st.max(1) + 1e-4, c + r + 1e-4])
    _check_layout(nodes, order, 540, pmin, pmax)
