"""Full scene query (object slots + BVH) and the edge-aware denoise on the GPU,
against golden vectors from the reference's scene_intersect and
edge_aware_denoise."""
import os

import numpy as np
import pytest

import golden_scenes as gs
import roxy_native as nat
from rendering.denoise import edge_aware_denoise, linear_to_display
from rendering.taichi.extractor import HostScene, build_device_scene
from test_host_logic import _ns

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("method", ["morton", "lbvh"])
def test_scene_intersect_matches_reference(method):
    g = np.load(os.path.join(GOLD, "trace_scene.npz"))
    world = gs.build_trace_scene(_ns())
    ds = build_device_scene(world, method=method)
    r = ds.native.intersect(g["si_ro"], g["si_rd"])
    # golden ids: object slot (is_bvh 0) or BVH-order triangle (is_bvh 1)
    bv = oracle_order(world)
    for i in range(len(g["si_t"])):
        ref_bvh = g["si_is_bvh"][i] == 1
        if g["si_idx"][i] < 0:
            assert r["kind"][i] == 0
            continue
        if ref_bvh:
            assert r["kind"][i] == 1 and r["id"][i] == bv[g["si_idx"][i]], i
        else:
            assert r["kind"][i] in (2, 3) and r["id"][i] == g["si_idx"][i], i
    hit = g["si_idx"] >= 0
    assert np.array_equal(r["t"][hit].view(np.uint32), g["si_t"][hit].view(np.uint32))
    np.testing.assert_allclose(r["normal"][hit], g["si_normal"][hit], atol=2e-7)


def oracle_order(world):
    from oracle import oracle
    b = HostScene(world).batch
    return oracle.bvh_build_morton(b.v0, b.v1, b.v2, 8)["order"]


def test_denoise_pass0_equals_reference_filter():
    g = np.load(os.path.join(GOLD, "denoise.npz"))
    for case in g["case_names"]:
        r, sc, amt = g[f"{case}/params"]
        kw = {k: g[f"{case}/{k}"] for k in ("normal", "albedo", "depth") if f"{case}/{k}" in g.files}
        out = edge_aware_denoise(g[f"{case}/pixels"], int(r), float(sc), float(amt), **kw)
        ref = g[f"{case}/out"]
        # float32 op order is the reference's; only expf's last bits differ
        np.testing.assert_allclose(out, ref, rtol=2e-6, atol=2e-6, err_msg=str(case))
    np.testing.assert_array_equal(linear_to_display(g["display/in"]), g["display/out"])


def test_denoise_reference_contracts():
    px = np.random.default_rng(1).random((4, 4, 3), dtype=np.float32)
    assert edge_aware_denoise(px, radius=0) is px
    assert edge_aware_denoise(px, amount=0.0) is px
    p = np.zeros((5, 5, 3), np.float32)
    p[:, :] = 0.2
    p[2, 2] = 1.0
    f = edge_aware_denoise(p, radius=1, sigma_color=0.2, amount=0.8)
    assert f.shape == p.shape and np.isfinite(f).all() and f[2, 2, 0] > f[0, 0, 0]
    with pytest.raises(ValueError, match="normal guide"):
        edge_aware_denoise(np.zeros((3, 5, 3), np.float32), normal=np.zeros((3, 4, 3), np.float32))
    base = np.zeros((3, 5, 3), np.float32)
    base[:, 2:] = 1.0
    un = edge_aware_denoise(base, radius=1, sigma_color=10.0, amount=1.0)
    nrm = np.zeros((3, 5, 3), np.float32)
    nrm[:, :2] = [0, 1, 0]
    nrm[:, 2:] = [0, -1, 0]
    gd = edge_aware_denoise(base, radius=1, sigma_color=10.0, amount=1.0, normal=nrm, sigma_normal=0.1)
    assert gd[1, 1, 0] < un[1, 1, 0] * 0.25 and gd[1, 2, 0] > un[1, 2, 0] + 0.2


def _atrous_numpy(src, normal, albedo, depth, passes, sc=0.08, sn=0.35, sa=0.2, sd=1.0, amount=0.8):
    """Plain numpy a-trous with the same kernel (taps 2^i apart, reflect)."""
    H, W = src.shape[:2]
    cur = src.astype(np.float64)
    s2 = [2 * max(s * s, 1e-8) for s in (sc, sn, sa, sd)]

    def refl(i, n):
        p = 2 * (n - 1)
        i = np.mod(i, p)
        return np.where(i >= n, p - i, i)

    yy, xx = np.mgrid[0:H, 0:W]
    for k in range(passes):
        step = 1 << k
        acc = np.zeros_like(cur)
        ws = np.zeros((H, W))
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                y2, x2 = refl(yy + dy * step, H), refl(xx + dx * step, W)
                w = 1.0 / (1 + dx * dx + dy * dy) * np.exp(-((cur[y2, x2] - cur) ** 2).sum(2) / s2[0])
                w *= np.exp(-((normal[y2, x2] - normal) ** 2).sum(2) / s2[1])
                w *= np.exp(-((albedo[y2, x2] - albedo) ** 2).sum(2) / s2[2])
                w *= np.exp(-((depth[y2, x2] - depth) ** 2) / s2[3])
                acc += cur[y2, x2] * w[:, :, None]
                ws += w
        cur = acc / np.maximum(ws, 1e-8)[:, :, None]
    return src * (1 - amount) + cur * amount


def test_atrous_five_passes_against_numpy():
    rng = np.random.default_rng(9)
    H, W = 45, 61
    src = rng.random((H, W, 3)).astype(np.float32)
    nrm = rng.normal(size=(H, W, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=2, keepdims=True)
    alb = rng.random((H, W, 3)).astype(np.float32)
    dep = (rng.random((H, W)) * 3 + 1).astype(np.float32)
    got = edge_aware_denoise(src, 1, 0.08, 0.8, normal=nrm, albedo=alb, depth=dep, passes=5)
    ref = _atrous_numpy(src, nrm, alb, dep, 5)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-5)


def test_denoise_edge_sizes():
    for H, W in ((1, 1), (1, 7), (6, 1), (2, 2), (17, 3)):
        px = np.random.default_rng(H * 31 + W).random((H, W, 3), dtype=np.float32)
        out = edge_aware_denoise(px, radius=2, sigma_color=0.3, amount=1.0, passes=3)
        assert out.shape == px.shape and np.isfinite(out).all()


def test_spheres_and_cubes_in_the_bvh_hit_as_the_linear_scan():
    """Spheres and cubes as BVH leaves return the same t (bit for bit),
    object slot and normal as the reference's linear object scan; planes
    stay linear."""
    ns = _ns()
    rng = np.random.default_rng(4)
    world = ns.World(use_sky=False, background_color=ns.Color(0.2, 0.2, 0.2))
    world.add_camera(ns.Camera(position=ns.Vec3(0, 2, 9), forward=ns.Vec3(0, -0.2, -1), up=ns.Vec3(0, 1, 0),
                               fov=50, width=64, height=64))
    for i in range(300):
        p = rng.uniform(-4, 4, 3)
        shape = ns.Cube(float(rng.uniform(0.1, 0.6))) if i % 2 else ns.Sphere(float(rng.uniform(0.05, 0.4)))
        world.add_object(ns.SceneObject(shape=shape, material=ns.Diffuse(ns.Color(0.5, 0.5, 0.5)),
                                        translation=ns.Vec3(*map(float, p)), name=f"o{i}"))
    world.add_object(ns.SceneObject(shape=ns.Plane(ns.Vec3(0, 1, 0), 4.5), material=ns.Diffuse(ns.Color(1, 1, 1)),
                                    name="floor"))
    ds = build_device_scene(world, method="lbvh")
    n = 40000
    ro = np.tile(np.array([[0.0, 2.0, 9.0]], np.float32), (n, 1)) + rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    rd = rng.normal(size=(n, 3)).astype(np.float32)
    rd[:, 2] = -np.abs(rd[:, 2]) - 0.5
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    ds.native.build_bvh(nat.RX_BVH_LBVH_SAH, 4, spheres_in_bvh=True)  # no triangles: built on request only
    in_bvh = ds.native.intersect(ro, rd)
    ds.native.build_bvh(nat.RX_BVH_LBVH_SAH, 4, spheres_in_bvh=False)
    linear = ds.native.intersect(ro, rd)
    hit = linear["kind"] != 0
    assert hit.mean() > 0.5
    assert np.array_equal(in_bvh["t"].view(np.uint32), linear["t"].view(np.uint32))
    assert np.array_equal(in_bvh["id"][hit], linear["id"][hit])
    assert np.array_equal(in_bvh["normal"][hit], linear["normal"][hit])
    objs = linear["kind"] == 3
    # 2: object in the BVH, 3: linear slot; only the plane (slot 300) stays linear
    plane = objs & (linear["id"] == 300)
    assert plane.any() and (objs & ~plane).any()
    assert (in_bvh["kind"][objs & ~plane] == 2).all() and (in_bvh["kind"][plane] == 3).all()
