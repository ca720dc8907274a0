"""Pins the CPU oracle to golden vectors produced by the reference's own code.

Every fixture under tests/golden/ was written by make_golden.py executing the
reference source; these tests need no GPU.
"""
import os

import numpy as np
import pytest

from oracle import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def test_bvh_build_matches_reference_builder_bit_exact():
    g = _load("bvh_build.npz")
    for case in g["case_names"]:
        c = {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith(f"{case}/")}
        out = oracle.bvh_build_morton(c["v0"], c["v1"], c["v2"], int(c["leaf"]))
        for key in ("left", "right", "start", "count", "order"):
            np.testing.assert_array_equal(out[key], c[key], err_msg=f"{case}:{key}")
        for key in ("node_min", "node_max"):
            assert np.array_equal(out[key].view(np.uint32), c[key].view(np.uint32)), f"{case}:{key}"


def _trav_scene(c):
    order = c["order"]
    return oracle.Scene(node_min=c["node_min"], node_max=c["node_max"], left=c["left"], right=c["right"],
                        start=c["start"], count=c["count"], v0=c["v0"][order], v1=c["v1"][order],
                        v2=c["v2"][order])


def test_traversal_matches_reference_bvh_intersect_bit_exact():
    g = _load("traversal.npz")
    for case in g["case_names"]:
        c = {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith(f"{case}/")}
        sc = _trav_scene(c)
        t, idx, u, v = oracle.bvh_intersect(sc, c["ro"], c["rd"])
        np.testing.assert_array_equal(idx, c["idx"], err_msg=case)
        hit = idx >= 0
        assert np.array_equal(t[hit].view(np.uint32), c["t"][hit].view(np.uint32))
        assert np.array_equal(u[hit].view(np.uint32), c["u"][hit].view(np.uint32))
        assert np.array_equal(v[hit].view(np.uint32), c["v"][hit].view(np.uint32))
        occ = oracle.bvh_occluded(sc, c["ro"], c["rd"], c["max_t"])
        np.testing.assert_array_equal(occ, c["occluded"], err_msg=case)


def test_primitive_intersections_match_reference():
    g = _load("prims.npz")
    n = len(g["ro"])
    objs_sph = dict(type=np.zeros(1, np.int32))
    # triangle KAT through the single-triangle entry
    t, _, _ = oracle.tri_intersect(g["ro"], g["rd"], g["v0"], g["v1"], g["v2"])
    assert np.array_equal(t.view(np.uint32), g["t_tri"].view(np.uint32))
    # spheres / planes / cubes through scene_intersect with one object each
    for kind, key in ((0, "t_sphere"), (1, "t_plane"), (2, "t_cube")):
        got = np.zeros(n, np.float32)
        for i in range(n):
            objs = dict(type=np.array([kind], np.int32), center=g["center"][i:i + 1],
                        radius=g["radius"][i:i + 1], normal=g["normal"][i:i + 1], offset=g["offset"][i:i + 1],
                        extra=g["half"][i:i + 1], v0=np.zeros((1, 3)), v1=np.zeros((1, 3)), v2=np.zeros((1, 3)),
                        mat_type=np.zeros(1), albedo=np.ones((1, 3)), roughness=np.zeros(1), ior=np.ones(1),
                        emission=np.zeros(1))
            sc = oracle.Scene(objects=objs)
            r = oracle.scene_intersect(sc, g["ro"][i:i + 1], g["rd"][i:i + 1])
            got[i] = r["t"][0] if r["idx"][0] >= 0 else -1.0
        ref = g[key].copy()
        ref[~(ref > 0.001)] = -1.0
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), key
    del objs_sph


def trace_scene_oracle(g, compat=True, extra_lights=None):
    objs = {k[4:]: g[k] for k in g.files if k.startswith("obj_")}
    nl = len(g["light_radius"])
    lights = dict(kind=np.zeros(nl, np.int32), p0=g["light_center"],
                  p1=np.stack([g["light_radius"], np.zeros(nl), np.zeros(nl)], 1),
                  p2=np.zeros((nl, 3)), albedo=g["light_albedo"], emission=g["light_emission"],
                  area=np.zeros(nl), pick_pdf=np.full(nl, 1.0 / max(nl, 1)), alias_prob=np.ones(nl),
                  alias_idx=np.arange(nl), obj=np.zeros(nl))
    return oracle.Scene(node_min=g["node_min"], node_max=g["node_max"], left=g["left"], right=g["right"],
                        start=g["start"], count=g["count"], v0=g["v0"], v1=g["v1"], v2=g["v2"], n0=g["n0"],
                        n1=g["n1"], n2=g["n2"], tri_mat=g["tri_mat"], mat_type=g["mat_type"],
                        mat_albedo=g["mat_albedo"], mat_roughness=g["mat_roughness"], mat_ior=g["mat_ior"],
                        mat_emission=g["mat_emission"], objects=objs, lights=lights)


def test_scene_intersect_matches_reference():
    g = _load("trace_scene.npz")
    sc = trace_scene_oracle(g)
    r = oracle.scene_intersect(sc, g["si_ro"], g["si_rd"])
    np.testing.assert_array_equal(r["idx"], g["si_idx"])
    np.testing.assert_array_equal(r["is_bvh"], g["si_is_bvh"])
    assert np.array_equal(r["t"].view(np.uint32), g["si_t"].view(np.uint32))
    np.testing.assert_allclose(r["normal"], g["si_normal"], rtol=0, atol=2e-7)


def test_trace_loop_matches_reference_trace_with_scripted_randoms():
    """oracle trace == reference trace() fed the same ti.random() stream."""
    g = _load("trace_scene.npz")
    sc = trace_scene_oracle(g)
    cfgs = g["tr_configs"]
    n = len(g["tr_cfg"])
    worst = 0.0
    for i in range(n):
        md, sky, mode, dlmd = (int(x) for x in cfgs[g["tr_cfg"][i]])
        p = oracle.make_params(64, 64, 1.0, 1.0, [0, 0, 0], [0, 0, -1], [1, 0, 0], [0, 1, 0], md, sky,
                               g["tr_bg"], direct_light_mode=mode, direct_light_max_depth=dlmd,
                               reference_compat=1)
        r = oracle.trace_scripted(sc, p, g["tr_ro"][i:i + 1], g["tr_rd"][i:i + 1], g["tr_stream"][i])
        assert r["consumed"] == g["tr_consumed"][i], i
        assert r["rays"] == g["tr_rays"][i], i
        for key in ("color", "normal", "albedo"):
            ref = g[f"tr_{key}"][i]
            err = np.max(np.abs(r[key] - ref) / (np.abs(ref) + 1e-3))
            worst = max(worst, err)
            assert err < 1e-4, (i, key, r[key], ref)
        assert abs(r["depth"] - g["tr_depth"][i]) <= 1e-6 * max(1.0, abs(g["tr_depth"][i]))
    assert worst < 1e-4


def texture_scene_oracle(g):
    textures = [g[f"tex{i}"] for i in range(len(g["tex_w"]))]
    return oracle.Scene(node_min=g["node_min"], node_max=g["node_max"], left=g["left"], right=g["right"],
                        start=g["start"], count=g["count"], v0=g["v0"], v1=g["v1"], v2=g["v2"], n0=g["n0"],
                        n1=g["n1"], n2=g["n2"], tri_mat=g["tri_mat"], mat_type=g["mat_type"],
                        mat_albedo=g["mat_albedo"], mat_roughness=g["mat_roughness"], mat_ior=g["mat_ior"],
                        mat_emission=g["mat_emission"],
                        objects={k[4:]: g[k] for k in g.files if k.startswith("obj_")},
                        lights=_golden_lights(g), uv0=g["uv0"], uv1=g["uv1"], uv2=g["uv2"], has_uv=g["has_uv"],
                        mat_texture=g["mat_texture"], textures=textures, tex_flip=g["tex_flip"])


def _golden_lights(g):
    nl = len(g["light_radius"])
    return dict(kind=np.zeros(nl, np.int32), p0=g["light_center"],
                p1=np.stack([g["light_radius"], np.zeros(nl), np.zeros(nl)], 1),
                p2=np.zeros((nl, 3)), albedo=g["light_albedo"], emission=g["light_emission"],
                area=np.zeros(nl), pick_pdf=np.full(nl, 1.0 / max(nl, 1)), alias_prob=np.ones(nl),
                alias_idx=np.arange(nl), obj=np.zeros(nl))


@pytest.mark.parametrize("name", ["texture_scene.npz", "texture_scene_indexed.npz"])
def test_texture_sampling_matches_reference(name):
    """_sample_texture and _bvh_albedo of the restatement equal the
    reference's float32 results bit for bit."""
    g = _load(name)
    sc = texture_scene_oracle(g)
    for t in range(len(g["tex_w"])):
        out = oracle.sample_texture(sc, t, g["st_uv"])
        assert np.array_equal(out.view(np.uint32), g["st_out"][t].view(np.uint32)), t
    n = len(g["tri_mat"])
    out = oracle.bvh_albedo(sc, np.arange(n), g["tri_mat"], g["ba_u"], g["ba_v"], g["mat_albedo"][g["tri_mat"]])
    assert np.array_equal(out.view(np.uint32), g["ba_out"].view(np.uint32))


@pytest.mark.parametrize("name", ["texture_scene.npz", "texture_scene_indexed.npz"])
def test_textured_trace_matches_reference_trace_with_scripted_randoms(name):
    g = _load(name)
    sc = texture_scene_oracle(g)
    cfgs = g["tr_configs"]
    for i in range(len(g["tr_cfg"])):
        md, sky, mode, dlmd = (int(x) for x in cfgs[g["tr_cfg"][i]])
        p = oracle.make_params(64, 64, 1.0, 1.0, [0, 0, 0], [0, 0, -1], [1, 0, 0], [0, 1, 0], md, sky,
                               g["tr_bg"], direct_light_mode=mode, direct_light_max_depth=dlmd,
                               reference_compat=1)
        r = oracle.trace_scripted(sc, p, g["tr_ro"][i:i + 1], g["tr_rd"][i:i + 1], g["tr_stream"][i])
        assert r["consumed"] == g["tr_consumed"][i], i
        assert r["rays"] == g["tr_rays"][i], i
        for key in ("color", "normal", "albedo"):
            ref = g[f"tr_{key}"][i]
            err = np.max(np.abs(r[key] - ref) / (np.abs(ref) + 1e-3))
            assert err < 1e-4, (i, key, r[key], ref)


def test_denoise_restatement_matches_reference():
    g = _load("denoise.npz")
    for case in g["case_names"]:
        r, sc, amt = g[f"{case}/params"]
        kw = {k: g[f"{case}/{k}"] for k in ("normal", "albedo", "depth") if f"{case}/{k}" in g.files}
        out = oracle.edge_aware_denoise(g[f"{case}/pixels"], int(r), float(sc), float(amt), **kw)
        np.testing.assert_array_equal(out, g[f"{case}/out"], err_msg=str(case))
    np.testing.assert_array_equal(oracle.linear_to_display(g["display/in"]), g["display/out"])


def test_philox_known_answer():
    # Random123 known-answer vectors for Philox4x32-10 (published with the paper's code)
    assert list(oracle.philox([0, 0, 0, 0], 0, 0)) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(oracle.philox([0xFFFFFFFF] * 4, 0xFFFFFFFF, 0xFFFFFFFF)) == \
        [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], 0xA4093822, 0x299F31D0)) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def _f64_bits_equal(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("name", ["obj_small", "obj_random"])
def test_obj_parse_restatement_matches_reference_reader(name):
    """oracle.obj_parse against OBJReader._parse_indexed run on the same text:
    float64 bits (inf / nan / -0.0 included), index tables, group names,
    used groups and the unrecognised-token warnings."""
    import json
    from oracle.obj_parse import parse_indexed
    g = _load(name + ".npz")
    meta = json.loads(bytes(g["meta"]).decode())
    r = parse_indexed(bytes(g["text"]))
    for k in ("positions", "normals", "uvs"):
        assert _f64_bits_equal(r[k], g[k]), k
    for k in ("tri_pos_idx", "tri_normal_idx", "tri_uv_idx", "tri_group_idx"):
        np.testing.assert_array_equal(r[k], g[k], err_msg=k)
    assert r["groups"] == meta["groups"]
    assert sorted(r["used_groups"]) == meta["mat_groups"]
    assert [f"Warning: Unrecognized OBJ token: {t!r}" for t in r["unknown"]] == meta["warnings"]
