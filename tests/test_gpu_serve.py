"""Serving with continuous batching (rx_serve_*): requests admitted while
others render produce the same image as rendering them alone (bit for
bit), admission respects the memory budget and the active-slot limit, a
request's preview arrives before its final image, and misuse is reported."""
import numpy as np
import pytest

import golden_scenes as gs
import roxy_native as nat
import workloads
from rendering.batch import Job
from rendering.serving import RenderServer, poisson_run
from test_host_logic import _ns

pytestmark = pytest.mark.gpu

BUFS = (nat.RX_ACC_RADIANCE, nat.RX_ACC_NORMAL, nat.RX_ACC_ALBEDO, nat.RX_ACC_DEPTH, nat.RX_ACC_DISPLAY)


def _jobs():
    ns = _ns()
    rng = np.random.default_rng(4)
    worlds = [workloads.cornell_box(32, 32), gs.build_trace_scene(ns), workloads.instanced_box_scene(2000, 3, 32, 32),
              gs.build_texture_scene(ns)]
    jobs = []
    for k in range(10):
        w = worlds[k % len(worlds)]
        W, H = int(rng.integers(16, 48)), int(rng.integers(16, 48))
        jobs.append(Job(w, W, H, int(rng.integers(1, 6)), int(rng.integers(2, 9)),
                        direct_light_mode=int(k % 3 == 0), direct_light_max_depth=int(rng.integers(1, 6)),
                        seed=100 + k).prepare())
    return jobs


def _solo(j):
    acc = nat.Accumulator(j.width, j.height)
    acc.render(j.scene.native, j.params, j.spp)
    return [acc.read(w) for w in BUFS]


def _check_same(server, rid, ref):
    for w, r in zip(BUFS, ref):
        got = server.read(rid, w)
        assert np.array_equal(got.view(np.uint32), r.view(np.uint32)), w


def test_served_requests_equal_solo_renders():
    jobs = _jobs()
    refs = [_solo(j) for j in jobs]
    srv = RenderServer(hbm_budget=8e9, max_active=4, step_paths=4000, wave_paths=1 << 16)
    ids = [srv.submit(j.scene.native, j.params, j.spp) for j in jobs]
    for rid, ref in zip(ids, refs):
        srv.wait(rid, final=True, timeout=60)
        info = srv.info(rid)
        assert info["state"] == "done" and info["frames_done"] == info["frames"]
        assert 0 <= info["t_admit"] <= info["t_preview"] <= info["t_final"]
        _check_same(srv, rid, ref)
        srv.release(rid)
    st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert 1 <= st["max_active_seen"] <= 4 and st["steps"] > 1
    srv.close()


def test_admission_respects_the_memory_budget():
    ns = _ns()
    worlds = [workloads.cornell_box(40, 40), gs.build_trace_scene(ns)]
    first = [Job(w, 40, 40, 3, 5, seed=200 + k).prepare() for k, w in enumerate(worlds)]
    jobs = first + [Job(worlds[k % 2], 40, 40, 3, 5, seed=200 + k, scene=first[k % 2].scene).prepare()
                    for k in range(2, 6)]
    # the wave state, both scenes and room for two and a half 40x40 accumulators
    base = (1 << 14) * (7 * 16 + 3 * 4 + 48)
    scenes = sum({id(j.scene.native): j.scene.native.device_bytes() for j in jobs}.values())
    acc = 40 * 40 * 64 + 64
    budget = base + scenes + int(2.5 * acc)
    srv = RenderServer(hbm_budget=budget, max_active=16, step_paths=1 << 14, wave_paths=1 << 14)
    ids = [(srv.submit(j.scene.native, j.params, j.spp), j) for j in jobs]
    for rid, j in ids:
        srv.wait(rid, final=True, timeout=60)
        _check_same(srv, rid, _solo(j))
        srv.release(rid)
    st = srv.stats()
    assert st["completed"] == len(jobs)
    assert st["max_active_seen"] == 2  # the third accumulator never fits
    assert st["max_bytes_in_use"] <= budget
    assert st["bytes_in_use"] == base  # everything but the wave state released
    srv.close()


def test_preview_before_final_and_errors():
    jobs = _jobs()
    big = Job(workloads.cornell_box(64, 64), 256, 256, 64, 8, direct_light_max_depth=8, seed=7).prepare()
    srv = RenderServer(hbm_budget=4e9, max_active=8, step_paths=256 * 256 * 2, wave_paths=1 << 20)
    rid = srv.submit(big.scene.native, big.params, big.spp)
    srv.wait(rid, final=False, timeout=60)
    info = srv.info(rid)
    assert info["frames_done"] >= 1 and info["t_preview"] > 0
    prev = srv.read(rid)
    assert prev.shape == (256, 256, 3) and np.isfinite(prev).all()
    # a second request queues behind the first (one active slot): releasing
    # it while it waits is an error
    one = RenderServer(hbm_budget=4e9, max_active=1, step_paths=1 << 20, wave_paths=1 << 20)
    a = one.submit(big.scene.native, big.params, big.spp)
    b = one.submit(big.scene.native, big.params, 1)
    with pytest.raises(nat.RxError, match="still being served"):
        one.release(b)
    one.wait(a, timeout=120)
    one.wait(b, timeout=120)
    one.release(a)
    one.release(b)
    one.close()
    srv.wait(rid, final=True, timeout=120)
    assert srv.info(rid)["frames_done"] == 64
    srv.release(rid)
    with pytest.raises(ValueError):
        srv.submit(jobs[0].scene.native, jobs[0].params, 0)
    with pytest.raises(ValueError):
        srv.info(rid)  # released
    tiny = RenderServer(hbm_budget=1 << 20, max_active=1, step_paths=1 << 10, wave_paths=1 << 10)
    with pytest.raises(AssertionError, match="exceeds"):
        tiny.submit(big.scene.native, big.params, 4)
    tiny.close()
    srv.close()


def test_poisson_run_reports_latencies():
    jobs = _jobs()
    srv = RenderServer(hbm_budget=8e9, max_active=8, step_paths=8000, wave_paths=1 << 16)
    r = poisson_run(srv, [(j.scene.native, j.params, j.spp) for j in jobs], rate=200.0, seed=1)
    assert r["requests"] == len(jobs)
    assert 0 < r["preview_p50_ms"] <= r["preview_p99_ms"] and r["preview_p50_ms"] <= r["final_p50_ms"]
    assert r["throughput_rps"] > 0
    assert srv.stats()["completed"] == len(jobs)
    srv.close()


def test_requests_with_scenes_built_on_arrival_equal_solo_renders():
    """Each request arrives as a world: its scene is extracted and its BVH
    built when it arrives, while earlier requests are rendering; the served
    image equals a solo render of the same world bit for bit, and the
    scenes' device memory is charged and given back with the requests.  The
    Poisson run builds each scene on the server's context under
    rx_ctx_hold (as the serving benchmark does); the image check builds
    them on a second context of the device."""
    import math

    from rendering.taichi.extractor import build_device_scene
    from rendering.taichi.trace import make_params
    worlds = [workloads.displaced_icosphere_scene(48, 27, subdiv=5, n_spheres=8, seed=3000 + k) for k in range(3)]
    specs = [(worlds[k % 3], 48 + 16 * (k % 2), 27 + 9 * (k % 2), 1 + k % 4, 100 + k) for k in range(8)]

    bctx = nat.Context(0)  # a second context of the device

    def request(world, W, H, spp, seed, own=False):
        def prepare():
            if own:  # on the server's context, holding its lock (as the serving bench builds)
                ctx = nat.context()
                with ctx.hold():
                    ds = build_device_scene(world, method="lbvh", ctx=ctx)
                    ds.use_lights(False)
            else:
                ds = build_device_scene(world, method="lbvh", ctx=bctx)
                ds.use_lights(False)
                bctx.sync()
            cam = world.active_camera
            p = make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, 12, int(world._use_sky), 0,
                            1, 10.0, list(world._background_color), list(cam.position), list(cam.forward),
                            list(cam.right), list(cam.up), seed=seed)
            return ds.native, p, spp, ds
        return prepare

    srv = RenderServer(hbm_budget=8e9, max_active=4, step_paths=3000, wave_paths=1 << 16)
    base = srv.stats()["bytes_in_use"]
    r = poisson_run(srv, [request(*s, own=True) for s in specs], rate=400.0, seed=3)
    assert r["requests"] == len(specs) and r["prepare_p50_ms"] > 0
    st = srv.stats()
    assert st["completed"] == len(specs) and st["failed"] == 0
    assert st["bytes_in_use"] == base
    srv.close()
    # served images of scenes built while earlier requests render, against
    # solo renders of the same scenes
    srv = RenderServer(hbm_budget=8e9, max_active=4, step_paths=3000, wave_paths=1 << 16)
    ids = []
    for s in specs:
        scene, p, spp, ds = request(*s)()
        ids.append((srv.submit(scene, p, spp), scene, p, spp, ds))
    for rid, scene, p, spp, _ in ids:
        srv.wait(rid, final=True, timeout=60)
        acc = nat.Accumulator(p.width, p.height, bctx)  # a solo render on the scene's own context
        acc.render(scene, p, spp)
        _check_same(srv, rid, [acc.read(w) for w in BUFS])
        srv.release(rid)
    srv.close()
