"""ORACLE — test infrastructure only.

Closest-hit parity check between the CUDA scene query (`rx_scene_intersect`)
and the oracle's `scene_intersect` (a restatement of
rendering/taichi/intersect.py:249-309 over the reference's own Morton tree).

The two traversals walk different trees (the product traverses an LBVH whose
leaves include the spheres and cubes; the oracle the reference's count-median
Morton tree plus its linear object scan), so they may legitimately pick
different primitives where two candidates are equally close.  Those rays are
excluded and counted, never silently accepted:

* edge rays: the hit lies within `edge_eps` (barycentric) of a triangle edge
  in either side's hit triangle (the neighbouring triangle across that edge
  is hit at the same t up to rounding);
* exact ties: the product's primitive, re-intersected by the oracle's own
  triangle test or object scan, gives bit-for-bit the oracle's t.

Every other ray must name the same primitive: the same triangle (caller
order) or the same object slot, or miss on both sides.  Matching hits are
then compared on t, u, v (relative `rtol`) and on the shading normal.

Only tests/ and the smoke check import this module.
"""
import numpy as np

from . import oracle


def reference_ids(ref, order):
    """Oracle scene_intersect result -> (is_tri, id) with triangle ids in the
    caller's order (`order` maps BVH order to caller order,
    bvh_builder.py:528-544) and object slots as themselves; id -1 = miss."""
    idx = ref["idx"]
    is_tri = (ref["is_bvh"] == 1) & (idx >= 0)
    ids = np.where(is_tri, order[np.maximum(idx, 0)], idx)
    ids = np.where(idx >= 0, ids, -1)
    return is_tri, ids.astype(np.int64)


def compare_closest(gpu, ref, order, ro, rd, v0, v1, v2, objects_scene=None, edge_eps=1e-6, rtol=1e-5):
    """gpu: rx_scene_intersect output (kind 0 miss, 1 triangle, 2 object in
    the BVH, 3 object in the linear scan; id; t; u; v; normal).  ref: oracle
    scene_intersect output.  v0..v2: caller-order triangle corners.
    objects_scene: an oracle.Scene holding only the object slots (used to
    re-intersect a product object hit), or None when there are no objects.

    Returns a dict of counts; raises AssertionError on any mismatch outside
    the exclusions or any disagreement in t / u / v / normal."""
    n = len(ro)
    r_tri, r_id = reference_ids(ref, order)
    g_kind = gpu["kind"]
    g_tri = g_kind == 1
    g_id = np.where(g_kind == 0, -1, gpu["id"]).astype(np.int64)
    same = (r_tri == g_tri) & (r_id == g_id)

    def bary_min(u, v):
        return np.minimum(np.minimum(u, v), 1.0 - u - v)

    near_edge = (r_tri & (bary_min(ref["u"], ref["v"]) < edge_eps)) | \
                (g_tri & (bary_min(gpu["u"], gpu["v"]) < edge_eps))
    ties = np.zeros(n, bool)
    cand = np.nonzero(~same & ~near_edge & (r_id >= 0) & (g_id >= 0))[0]
    if len(cand):
        tri_c = cand[g_tri[cand]]
        if len(tri_c):
            k = g_id[tri_c]
            tt, _, _ = oracle.tri_intersect(ro[tri_c], rd[tri_c], v0[k], v1[k], v2[k])
            ties[tri_c] = tt.view(np.uint32) == ref["t"][tri_c].view(np.uint32)
        obj_c = cand[~g_tri[cand]]
        if len(obj_c) and objects_scene is not None:
            o = oracle.scene_intersect(objects_scene, ro[obj_c], rd[obj_c])
            ties[obj_c] = (o["idx"] == g_id[obj_c]) & \
                          (o["t"].view(np.uint32) == ref["t"][obj_c].view(np.uint32))
    excluded = ~same & (near_edge | ties)
    bad = ~same & ~excluded
    if bad.any():
        i = np.nonzero(bad)[0][:8]
        raise AssertionError(f"{int(bad.sum())} closest-hit id mismatches outside exclusions of {n} rays; "
                             f"rays {i.tolist()}: gpu kind/id {g_kind[i].tolist()}/{g_id[i].tolist()}, "
                             f"oracle tri/id {r_tri[i].tolist()}/{r_id[i].tolist()}")
    hit = same & (r_id >= 0)
    np.testing.assert_allclose(gpu["t"][hit], ref["t"][hit], rtol=rtol, err_msg="hit distance")
    th = hit & r_tri
    np.testing.assert_allclose(gpu["u"][th], ref["u"][th], rtol=rtol, atol=rtol * 0.1, err_msg="barycentric u")
    np.testing.assert_allclose(gpu["v"][th], ref["v"][th], rtol=rtol, atol=rtol * 0.1, err_msg="barycentric v")
    np.testing.assert_allclose(gpu["normal"][hit], ref["normal"][hit], atol=1e-5, err_msg="shading normal")
    return dict(rays=n, hits=int((r_id >= 0).sum()), triangle_hits=int(r_tri.sum()),
                object_hits=int(((r_id >= 0) & ~r_tri).sum()), matched=int(same.sum()),
                excluded_edge=int((~same & near_edge).sum()), excluded_ties=int((~same & ties & ~near_edge).sum()),
                edge_rays=int(near_edge.sum()),
                t_bit_exact=bool(np.array_equal(gpu["t"][hit].view(np.uint32), ref["t"][hit].view(np.uint32))))
