"""Benchmark: Mrays/s of the path-tracing hot path on one B200 per rank.

Workload (default "icosphere"): the 327,680-triangle displaced icosphere with
64 analytic spheres, one emissive quad and uniform background radiance 0.2,
rendered at 1920 x 1080, 64 samples per pixel, max depth 12, FP32.  A step is
one full 64-spp render of that frame (BVH resident; the accumulators reset
each step).  Rays are counted as the reference counts them: one per bounce
including the primary ray, one per shadow ray.

  value  rays / second with the scene resident in HBM (device time, max over
         ranks, CUDA events on the library's stream)
  e2e    the same metric through TaichiRenderer.render(): host scene arrays
         copied to the device, GPU BVH build, the 64-spp render, and the
         display image copied back, every step

Multi-GPU: the path does not need an exchange; each rank renders its own
replica of the frame ("replicas only") and value is the sum of rays over
ranks divided by the slowest rank's time.

`--impl reference` times the CPU restatement of the reference's Taichi path
(the oracle, C++/OpenMP on all host cores) on a bounded sample of the same
workload; the reference's Taichi runtime is not installable here.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# paths per wavefront when rx_render_params.wave_paths is 0 (rx_render.cu
# picks 2^27 on a B200: the largest size whose state fits in a quarter of
# the free memory); used to count extend launches per step
WAVE_PATHS = 1 << 27
sys.path[:0] = [os.path.join(ROOT, "roxy-dcc_b200"), ROOT]

import numpy as np  # noqa: E402

WORKLOADS = {
    "icosphere": dict(width=1920, height=1080, spp=64, max_depth=12, dlmd=1,
                      desc="displaced icosphere 327,680 tris + 64 spheres, 1920x1080, 64 spp, depth 12"),
    "cornell": dict(width=256, height=256, spp=16, max_depth=8, dlmd=8, denoise_passes=5,
                    desc="Cornell box 36 tris, 256x256, 16 spp, depth 8, NEE every bounce, "
                         "then the 5-pass a-trous denoise"),
    # same scene at 640x360 / 16 spp: the kernel-profiling case (same kernels,
    # one wave of 3.7M paths, < 1 GB on the device)
    "icosphere-small": dict(width=640, height=360, spp=16, max_depth=12, dlmd=1,
                            desc="displaced icosphere 327,680 tris + 64 spheres, 640x360, 16 spp, depth 12"),
}


def _world(name):
    import workloads
    if name == "icosphere":
        return workloads.displaced_icosphere_scene()
    if name == "icosphere-small":
        return workloads.displaced_icosphere_scene(640, 360)
    return workloads.cornell_box()


def _params(world, w, make_params, seed=0):
    cam = world.active_camera
    return make_params(w["width"], w["height"], math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio,
                       w["max_depth"], int(world._use_sky), 0, w["dlmd"], 10.0, list(world._background_color),
                       list(cam.position), list(cam.forward), list(cam.right), list(cam.up), seed=seed)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_baseline(wname, world, seconds_target=15.0, rows=None, spp=None):
    """Oracle (C++/OpenMP) on a row-stratified sample of the workload: bands of
    rows spaced evenly over the frame, spp sized to a bounded CPU time."""
    from oracle import oracle
    from rendering.taichi.extractor import HostScene, slot_arrays
    w = WORKLOADS[wname]
    h = HostScene(world)
    b = h.batch
    bvh = oracle.bvh_build_morton(b.v0, b.v1, b.v2, 8)
    o = bvh["order"]
    lights = dict(h.lights(False))
    lights["obj"] = np.zeros(len(lights["kind"]), np.int32)
    pt, pa, pr, pi, pe = h.palette
    sc = oracle.Scene(node_min=bvh["node_min"], node_max=bvh["node_max"], left=bvh["left"], right=bvh["right"],
                      start=bvh["start"], count=bvh["count"], v0=b.v0[o], v1=b.v1[o], v2=b.v2[o], n0=b.n0[o],
                      n1=b.n1[o], n2=b.n2[o], tri_mat=h.mat_idx[o], mat_type=pt, mat_albedo=pa, mat_roughness=pr,
                      mat_ior=pi, mat_emission=pe, objects=slot_arrays(h.slots) if h.slots else None, lights=lights)
    cam = world.active_camera
    p = oracle.make_params(w["width"], w["height"], math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio,
                           list(cam.position), list(cam.forward), list(cam.right), list(cam.up), w["max_depth"],
                           int(world._use_sky), list(world._background_color), direct_light_mode=0,
                           direct_light_max_depth=w["dlmd"], sample_clamp=10.0, reference_compat=0, seed=0)
    cores = os.cpu_count() or 1
    H = w["height"]
    # calibrate on 8 rows at 1 spp spread over the frame, then size the
    # sample to ~seconds_target: `bands` bands of rows spaced evenly from top
    # to bottom (row-stratified, so sky, mesh and spheres enter in the
    # frame's own proportions), each band's rows contiguous
    bands = min(16, H)
    t0 = time.perf_counter()
    for k in range(8):
        y = (2 * k + 1) * H // 16
        oracle.render(sc, p, 1, rows=(y, y + 1), n_threads=cores)
    per_row_spp = max(time.perf_counter() - t0, 1e-3) / 8.0
    fixed = rows is not None
    if rows is None:
        budget_rows_spp = seconds_target / per_row_spp
        spp = spp or max(1, min(w["spp"], int(budget_rows_spp // (4 * bands)) or 1))
        rows = int(max(bands, min(H, budget_rows_spp / spp)))
    for _ in range(4):
        rows = max(bands, min(H, rows))
        per_band = rows // bands
        starts = [max(0, min(H - per_band, (2 * k + 1) * H // (2 * bands) - per_band // 2)) for k in range(bands)]
        rays, dt = 0, 0.0
        for y0 in starts:
            t0 = time.perf_counter()
            rays += oracle.render(sc, p, spp, rows=(y0, y0 + per_band), n_threads=cores)["rays"]
            dt += time.perf_counter() - t0
        # the calibration rows carry per-call overhead: grow the sample
        # (rows first, then spp) until it takes about seconds_target
        if fixed or dt >= 0.6 * seconds_target or (rows >= H and spp >= w["spp"]):
            break
        grow = min(8.0, seconds_target / max(dt, 1e-3))
        if rows < H:
            rows = int(min(H, rows * grow))
        else:
            spp = int(min(w["spp"], max(spp + 1, spp * grow)))
    rows = per_band * bands
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "port",
            "sample": f"{bands} bands of {per_band} rows spaced evenly over the {w['width']}x{H} frame "
                      f"({rows} rows), {spp} spp, depth {w['max_depth']} ({rays} rays in {dt:.2f} s)",
            "seconds": dt, "rays": rays}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    if args.workload in ("batch", "serve", "denoiser"):
        print(json.dumps({"impl": "reference", "unavailable": "the batched and serving workloads' baseline is the "
                                                              "plain one-scene-at-a-time GPU path in their own line"}))
        return 0
    world = _world(args.workload)
    w = WORKLOADS[args.workload]
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(args.workload, world, seconds_target=max(2.0, 60.0 / max(args.steps + args.warmup, 1)))
        if i >= args.warmup:
            vals.append(cb)
    v = statistics.mean(c["value"] for c in vals)
    ms = statistics.mean(c["seconds"] for c in vals) * 1e3
    line = {"impl": "reference", "metric": "Mrays/s", "value": v, "unit": "Mrays/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": w["desc"], "impl_note": "CPU restatement of the reference Taichi path "
                                                           "(oracle, C++/OpenMP); Taichi is not installable"
                                                           + ("; times the trace only: the reference has no "
                                                              "multi-pass a-trous filter" if w.get("denoise_passes")
                                                              else "")},
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": vals[0]["cores"], "kind": "port",
                             "sample": vals[0]["sample"]},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import roxy_native as nat
    from rendering.image import Image
    from rendering.taichi.extractor import build_device_scene
    from rendering.taichi.trace import make_params
    from rendering.taichi_renderer import TaichiRenderer

    ws, rank, local = _dist()
    dist = None
    if ws > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = tdist
    import torch
    dev = local if ws > 1 else 0
    ctx = nat.context(dev)
    w = WORKLOADS[args.workload]
    world = _world(args.workload)
    W, H = w["width"], w["height"]

    # -- device-resident throughput -------------------------------------------
    t_build0 = time.perf_counter()
    ds = build_device_scene(world, method="lbvh")
    ds.use_lights(False)
    ctx.sync()
    build_s = time.perf_counter() - t_build0
    params = _params(world, w, make_params)
    acc = nat.Accumulator(W, H, ctx)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", dev))
    # Frames are queued back to back (asynchronous accumulator): the timed
    # region holds no host round trip; the device error bits of all timed
    # frames are checked by the ctx.sync() after it.
    acc.set_async(True)
    dn_passes = w.get("denoise_passes", 0)
    dn_params = nat.DenoiseParams(1, max(dn_passes, 5), 0.08, 0.35, 0.20, 1.0, 0.8, 1, 1, 1, 1)

    def step():
        acc.reset()
        acc.render(ds.native, params, w["spp"])
        if dn_passes:
            acc.denoise(dn_params, out=False)

    for _ in range(args.warmup):
        step()
    ctx.sync()
    launches = 0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ctx.sync()
    with ClockSampler(dev) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
            launches += acc.last_timing()["launches"] + dn_passes
        ev1.record(stream)
        ev1.synchronize()
    ctx.sync()
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    acc.set_async(False)
    rays_timed = acc.info()["rays"]  # the last timed frame's
    # Per-kernel split: the same frames again with CUDA events around every
    # launch (untimed for the headline); each frame must trace exactly the
    # rays the timed frames traced (same seeds, same frame base).
    acc.set_timing(True)
    kern = {"extend_ms": 0.0, "shade_ms": 0.0, "connect_ms": 0.0, "other_ms": 0.0, "accumulate_ms": 0.0}
    step_rays = []
    for _ in range(args.steps):
        acc.reset()
        acc.render(ds.native, params, w["spp"])
        tm = acc.last_timing()
        for k in kern:
            kern[k] += tm[k]
        step_rays.append(acc.info()["rays"])
    acc.set_timing(False)
    if any(r != rays_timed for r in step_rays):
        raise RuntimeError(f"frames traced different ray counts: {rays_timed} timed, {step_rays} split")
    total_rays = sum(step_rays)
    extend_rays = 0
    if dist:
        t = torch.tensor([ms], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        r = torch.tensor([float(total_rays)], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(r)
        total_rays = int(r.item())
    value = total_rays / (ms / 1e3) / 1e6

    # -- roofline of the dominant kernel (traversal) ----------------------------
    peak, peak_kind = _peaks()
    per_step = step_rays[0] if step_rays else 0
    n_shadow_est = None
    ext_ms = kern["extend_ms"] / max(args.steps, 1)
    shade_ms = kern["shade_ms"] / max(args.steps, 1)
    # extend rays per step = rays minus shadow rays; both counters come from
    # the device; shadow rays are at most one per diffuse bounce below dlmd
    stats = _ray_split(ds, acc, params, w)
    ext_rays = stats["extend_rays"]
    # algorithmic bytes of the closest-hit items: 40 B per ray (origin and
    # direction in, hit record out), 16 B for a camera ray, which bounce 0
    # makes in the kernel (only its hit record is written)
    cam_rays = W * H * w["spp"]
    ext_bytes = 40.0 * max(ext_rays - cam_rays, 0) + 16.0 * min(cam_rays, ext_rays)
    ext_gbs = ext_bytes / (ext_ms / 1e3) / 1e9 if ext_ms > 0 else 0.0
    # k_shade: 272 B per ray, less the 48 B of ray state a camera ray does
    # not read at bounce 0.  64 B of it (the hit triangle's normals and
    # palette index, the material record) come from the scene, which stays
    # in L2; the rest is path state streamed through HBM.
    shade_bytes = 272.0 * ext_rays - 48.0 * min(cam_rays, ext_rays)
    shade_gbs = shade_bytes / (shade_ms / 1e3) / 1e9 if shade_ms > 0 else 0.0
    shade_hbm = shade_bytes - 64.0 * ext_rays
    shade_hbm_gbs = shade_hbm / (shade_ms / 1e3) / 1e9 if shade_ms > 0 else 0.0
    # DRAM bytes per k_extend launch: ncu's DRAM bytes per closest-hit ray
    # (committed summary: one-pass DRAM counters over the 12 extend launches
    # of this frame) times the average rays per launch here (max_depth
    # launches per wave)
    spf = max(1, min(w["spp"], WAVE_PATHS // (W * H)))
    ext_launches = w["max_depth"] * -(-w["spp"] // spf)
    measured = _traffic()
    traffic = measured["k_extend"] * ext_rays / ext_launches if "k_extend" in measured else None
    shade_dram = measured.get("k_shade")

    # k_accumulate: one launch folds the wave's frames; per pixel it reads
    # each frame's sample radiance and first-hit guides (3 x 16 B) and reads
    # (3 x 16 B) and writes (4 x 16 B, display included) the running means
    acc_ms = kern["accumulate_ms"] / max(args.steps, 1)
    acc_bytes = W * H * (48.0 * w["spp"] + 112.0)
    acc_gbs = acc_bytes / (acc_ms / 1e3) / 1e9 if acc_ms > 0 else 0.0
    atrous = _atrous_roofline(nat, acc, stream, dn_params, W, H, peak, dev)

    # -- image error of the timed render against a float64 high-spp render ------
    quality = None
    if args.ref_spp > 0:
        from rendering.quality import reference_render, rel_mse
        t_ref = time.perf_counter()
        ref = reference_render(ds.native, params, args.ref_spp, ctx=ctx)
        quality = {"relmse": rel_mse(acc.read(nat.RX_ACC_RADIANCE), ref), "spp": w["spp"],
                   "ref_spp": args.ref_spp, "ref": "float64-accumulated render, independent seed, same clamp",
                   "ref_render_s": time.perf_counter() - t_ref}
        # the same frame with power-heuristic MIS (not the timed estimator)
        pm = nat.RenderParams.from_buffer_copy(params)
        pm.mis = 1
        acc_m = nat.Accumulator(W, H)
        acc_m.render(ds.native, pm, w["spp"])
        quality["relmse_mis"] = rel_mse(acc_m.read(nat.RX_ACC_RADIANCE), ref)
        del acc_m

    # -- end to end through TaichiRenderer ------------------------------------
    img = Image(W, H)
    r = TaichiRenderer(world, img, None, samples=w["spp"], max_depth=w["max_depth"],
                       direct_light_max_depth=w["dlmd"], denoise=bool(dn_passes),
                       denoise_passes=max(dn_passes, 1))
    r.render()  # warm: wave buffers, graph
    r.render()
    e2e_times, e2e_rays = [], []
    for _ in range(max(1, min(args.steps, 5))):
        ctx.sync()
        t0 = time.perf_counter()
        r.render()
        ctx.sync()
        e2e_times.append(time.perf_counter() - t0)
        e2e_rays.append(r.last_ray_count)
    h2d = int(r._scene.h2d_bytes + len(r._scene.slots) * 96)
    d2h = W * H * 3 * 4
    # wall-clock frames see host stalls (thread scheduling, the allocator):
    # the line reports the median frame and, beside it, the mean over all
    e2e_mean = sum(e2e_rays) / sum(e2e_times) / 1e6
    e2e_val = statistics.median(e2e_rays) / statistics.median(e2e_times) / 1e6
    if dist:
        t = torch.tensor([e2e_val], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(t)
        e2e_val = float(t.item())

    if rank == 0:
        cb = cpu_baseline(args.workload, world, seconds_target=15.0) if ws == 1 and not args.no_cpu else None
        line = {"metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / max(args.steps, 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator, no dataset)",
                "config": {"workload": w["desc"], "parallelism": f"replicas x{ws}",
                           "rays_per_step": per_step, "paths_per_step": W * H * w["spp"],
                           "paths_per_s": W * H * w["spp"] * args.steps * ws / (ms / 1e3),
                           "bvh": "LBVH + SAH collapse, leaf 4", "bvh_build_s_host_incl": build_s,
                           "l2": "wavefront state > L2 each wave; BVH + triangles L2-resident by design"},
                "gpu_launches": launches,
                "roofline": {"bound": "hbm", "kernel": "k_extend (closest-hit traversal) + k_tail",
                             "achieved": ext_gbs, "peak": peak, "unit": "GB/s", "frac": ext_gbs / peak,
                             "traffic": traffic, "peak_source": peak_kind,
                             "algorithmic_bytes_per_ray": ext_bytes / max(ext_rays, 1),
                             "note": f"traversal is latency/L2 bound; frac is of the {peak_kind} HBM copy bandwidth; "
                                     "extend time includes k_tail, which runs the last bounces of each wave "
                                     "(their traversal and shading) once the queue is short",
                             "extend_ms_per_step": ext_ms, "extend_rays_per_step": ext_rays,
                             "shade": {"achieved": shade_gbs, "frac": shade_gbs / peak,
                                       "algorithmic_bytes_per_ray": shade_bytes / max(ext_rays, 1),
                                       "ms_per_step": shade_ms,
                                       "hbm_streamed": {"achieved": shade_hbm_gbs, "frac": shade_hbm_gbs / peak,
                                                        "bytes_per_ray": shade_hbm / max(ext_rays, 1),
                                                        "note": "algorithmic bytes less the 64 B per ray read "
                                                                "from the L2-resident scene"},
                                       "dram_bytes_per_ray_small_case": shade_dram},
                             "accumulate": {"achieved": acc_gbs, "frac": acc_gbs / peak, "ms_per_step": acc_ms,
                                            "algorithmic_bytes_per_step": acc_bytes,
                                            "bytes": "per pixel 48 B x spp sample reads + 112 B running means"},
                             "atrous": atrous,
                             # the rest of a step: generate + accumulate (+ a
                             # separate shadow launch); and the timed step
                             # minus all kernel spans of the split pass (the
                             # reset memsets and launch gaps)
                             "other_ms_per_step": (kern["other_ms"] + kern["connect_ms"]) / max(args.steps, 1),
                             "gap_ms_per_step": (ms - sum(kern.values())) / max(args.steps, 1)},
                "clocks": clocks.summary(),
                "quality": quality,
                "e2e": {"value": e2e_val, "unit": "Mrays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "frames": len(e2e_times), "stat": "median frame", "mean_over_frames": e2e_mean,
                        "frame_ms": [round(t * 1e3, 3) for t in e2e_times],
                        "path": "TaichiRenderer.render(): extract + H2D + GPU BVH build + render"
                                + (f" + {dn_passes}-pass a-trous" if dn_passes else "") + " + D2H image"},
                "cpu_baseline": cb and {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _traffic():
    """DRAM bytes per unit of the hot kernels, from the committed ncu
    summaries (profiles/traffic.json: captured on the 640x360 16-spp case of
    the benchmark scene, per closest-hit ray for k_extend, per shaded ray
    for k_shade)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return {k: float(v["bytes_per_unit"]) for k, v in json.load(f).items()}
    except (OSError, ValueError, KeyError, TypeError):
        return {}


def _atrous_roofline(nat, acc, stream, dp, W, H, peak, dev, iters=10):
    """The edge-aware a-trous filter (all guides, radius 1, dp.passes passes)
    on the resident accumulators, each call timed alone with CUDA events on
    the library stream after a 256 MB write that evicts L2.  Algorithmic
    bytes: 52 B per pixel per pass (colour 12 + normal 12 + albedo 12 +
    depth 4 read, 12 written)."""
    import torch
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{dev}")
    times = []
    with torch.cuda.stream(stream):
        for i in range(iters + 3):
            flush.fill_(float(i))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            acc.denoise(dp, out=False)
            e1.record(stream)
            e1.synchronize()
            if i >= 3:
                times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    alg = 52.0 * W * H * dp.passes
    gbs = alg / (ms / 1e3) / 1e9
    return {"achieved": gbs, "frac": gbs / peak, "ms": ms, "passes": dp.passes, "pixels": W * H,
            "ms_per_pass": ms / dp.passes, "algorithmic_bytes": alg,
            "layout_bytes_per_pixel_pass": 64, "l2": "flushed (256 MB write) before each timed call"}


def _ray_split(ds, acc, params, w):
    """Extend (bounce) rays vs shadow rays of one render, from a separate
    instrumented frame with NEE disabled and enabled."""
    import copy

    import roxy_native as nat
    p2 = copy.copy(params)
    p2.direct_light_max_depth = 0
    tmp = nat.Accumulator(w["width"], w["height"], acc.ctx)
    tmp.render(ds.native, p2, w["spp"])
    ext = tmp.info()["rays"]
    tmp.close()
    return {"extend_rays": ext}


def run_batch(args):
    """Batched configuration: 64 seeded instanced-box scenes (1k-2M
    triangles, 256^2-1024^2, 1-64 spp, depth 4-16) rendered as one batch
    (rx_batch_*, autotuned) against the plain path, which renders the same
    jobs one scene at a time (rx_render per scene)."""
    import roxy_native as nat
    import torch
    import workloads
    from rendering.batch import BatchRenderer, Job

    ws, rank, local = _dist()
    dist = None
    dev = local if ws > 1 else 0
    if ws > 1:
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = tdist
    ctx = nat.context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", dev))
    specs = workloads.batch_specs(n_scenes=args.scenes)
    t0 = time.perf_counter()
    jobs = [Job(workloads.instanced_box_scene(s["n_tris"], s["seed"], s["width"], s["height"]), s["width"],
                s["height"], s["spp"], s["max_depth"], direct_light_max_depth=s["max_depth"], seed=s["seed"])
            for s in specs]
    br = BatchRenderer(jobs, ctx=ctx)
    ctx.sync()
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    cfg = br.autotune()
    tune_s = time.perf_counter() - t0

    def timed(fn):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ctx.sync()
        ev0.record(stream)
        fn()
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1)

    def reset_all():
        for j in jobs:
            j.acc.reset()

    # plain path: one scene at a time, one accumulator per resolution
    plain_acc = {}
    for j in jobs:
        if (j.width, j.height) not in plain_acc:
            plain_acc[(j.width, j.height)] = nat.Accumulator(j.width, j.height, ctx)

    def plain():
        rays = 0
        for j in jobs:
            a = plain_acc[(j.width, j.height)]
            a.reset()
            a.render(j.scene.native, j.params, j.spp)
            rays += a.info()["rays"]
        return rays

    for _ in range(args.warmup):
        reset_all()
        br.render()
        plain()
    if dist:
        dist.barrier()
    batch_ms, plain_ms, e2e_ms, rays = [], [], [], 0
    launches = 0
    with ClockSampler(dev) as clocks:
        for _ in range(args.steps):
            reset_all()
            batch_ms.append(timed(br.render))
            launches = br.batch.last_stats()["launches"]
    rays = sum(j.acc.info()["rays"] for j in jobs)
    for _ in range(args.steps):
        plain_ms.append(timed(plain))
    plain_rays = plain()

    # first previews: one frame of every scene, batched vs one at a time
    def plain_preview():
        for j in jobs:
            a = plain_acc[(j.width, j.height)]
            a.reset()
            a.render(j.scene.native, j.params, 1)

    def batch_preview():
        br.render(frames=1)

    for _ in range(2):
        reset_all()
        batch_preview()
        plain_preview()
    prev_b, prev_p = [], []
    for _ in range(args.steps):
        reset_all()
        prev_b.append(timed(batch_preview))
        prev_p.append(timed(plain_preview))
    # end to end: batch render plus read-back of every display image
    d2h = 0
    for _ in range(max(1, min(args.steps, 3))):
        reset_all()
        t = time.perf_counter()
        br.render()
        d2h = sum(j.acc.read(nat.RX_ACC_DISPLAY).nbytes for j in jobs)
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    ms = sum(batch_ms) / len(batch_ms)
    pms = sum(plain_ms) / len(plain_ms)
    if dist:
        t = torch.tensor([ms, pms], device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, pms = float(t[0]), float(t[1])
    n = len(jobs)
    if rank == 0:
        line = {"metric": "scenes/s", "value": n * ws / (ms / 1e3), "unit": "scenes/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded generator, no dataset)",
                "config": {"workload": f"{n} instanced-box scenes, {sum(s['n_tris'] for s in specs):,} tris, "
                                       "256^2-1024^2, 1-64 spp, depth 4-16 (seeded)",
                           "paths_per_step": sum(j.paths for j in jobs), "parallelism": f"replicas x{ws}",
                           "scene_build_s": build_s, "autotune_s": tune_s,
                           "tuned": {"wave_paths": cfg.wave_paths, "extend_block": cfg.extend_block,
                                     "leaf_size": cfg.leaf_size},
                           "l2": "wavefront state > L2"},
                "mrays_per_s": rays * ws / (ms / 1e3) / 1e6,
                "plain": {"ms_per_step": pms, "scenes_per_s": n * ws / (pms / 1e3),
                          "mrays_per_s": plain_rays * ws / (pms / 1e3) / 1e6,
                          "path": "rx_render one scene after another, scenes resident"},
                "speedup_vs_plain": pms / ms,
                "preview_1spp": {"batch_ms": sum(prev_b) / len(prev_b), "plain_ms": sum(prev_p) / len(prev_p),
                                 "batch_scenes_per_s": n * ws / (sum(prev_b) / len(prev_b) / 1e3),
                                 "plain_scenes_per_s": n * ws / (sum(prev_p) / len(prev_p) / 1e3),
                                 "speedup": sum(prev_p) / sum(prev_b)},
                "gpu_launches": launches, "clocks": clocks.summary(),
                "quality": {"equal_to_plain": "bit-identical images (tests/test_gpu_batch.py), so equal relMSE"},
                "e2e": {"value": n * ws / (sum(e2e_ms) / len(e2e_ms) / 1e3), "unit": "scenes/s",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
                        "path": "BatchRenderer.render() + read-back of every display image; scenes resident"}}
        print(json.dumps(line))
    br.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_denoiser(args):
    """Learned-denoiser configuration: the committed weights (trained on
    renderer-generated 4-spp / 256-spp pairs of other large-mesh scenes)
    denoise a 4-spp 1920x1080 render of the benchmark scene; relMSE of the
    noisy image, the 5-pass a-trous filter and the learned denoiser against a
    float64 4096-spp render; inference timed with CUDA events."""
    import roxy_native as nat
    import workloads
    from rendering.learned_denoiser import Denoiser, evaluate, evaluate_held_out, load_weights

    ws, rank, local = _dist()
    if rank != 0:
        return 0
    nat.context(0)
    net = Denoiser(weights=load_weights())
    with ClockSampler(0) as clocks:
        r = evaluate(net, workloads.displaced_icosphere_scene(), ref_spp=args.ref_spp or 4096)
    held = evaluate_held_out(net, ref_spp=args.ref_spp or 4096)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("bf16_tflops", 1590.0))
    line = {"metric": "frames/s", "value": 1e3 / r["infer_ms"], "unit": "frames/s", "n_gpus": 1, "steps": 10,
            "warmup": 3, "ms_per_step": r["infer_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 (fp32 accumulate)", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": "learned denoiser, 3-level U-Net 32/64/128, 1920x1080 4-spp render of the "
                                   "displaced-icosphere scene", "flops_per_frame": r["flops_per_frame"]},
            "roofline": {"bound": "tensor",
                         "kernel": "whole inference: k_conv_fwd_ws (tcgen05; 9 layers in one launch, e3b and d2a, "
                                   "whose weights do not fit beside the row ring in one, as two launches over "
                                   "the halves of their input channels) + pool / upsample / feature / output "
                                   "kernels; network FLOPs over the inference time",
                         "achieved": r["infer_tflops"], "peak": peak, "unit": "TFLOP/s",
                         "frac": r["infer_tflops"] / peak,
                         "peak_source": "measured" if "bf16_tflops" in peaks else "fallback", "traffic": None},
            "quality": {k: r[k] for k in ("relmse_noisy", "relmse_atrous", "relmse_learned", "spp", "ref_spp")}
            | {"held_out_mean": held["mean"], "held_out_views": held["views"],
               "held_out": "one orbit view of each of 8 scene seeds never rendered for training, 1920x1080"},
            "clocks": clocks.summary()}
    print(json.dumps(line))
    return 0


OBJ_KERNELS_PER_PARSE = 31  # line count + 3 scan kernels, line write, classify + 3, list, gather lines,
#                             6 channel scans x 3, gather prefix, emit


def _obj_sample(text, nbytes):
    """A prefix of the OBJ text ending at a line boundary."""
    cut = text.rfind(b"\n", 0, nbytes)
    return text[:cut + 1] if cut > 0 else text


def _obj_cpu_baseline(text, seconds_target=12.0):
    """The CPU restatement of OBJReader._parse_indexed (oracle.obj_parse) on a
    prefix of the workload sized to about `seconds_target` of work."""
    from oracle.obj_parse import parse_indexed
    size, t = 1 << 20, 0.0
    while True:
        sample = _obj_sample(text, size)
        t0 = time.perf_counter()
        parse_indexed(sample)
        t = time.perf_counter() - t0
        if t >= seconds_target / 4 or len(sample) == len(text):
            break
        size = int(size * min(8.0, max(2.0, seconds_target / 4 / max(t, 1e-3))))
    return {"value": len(sample) / 1e6 / t, "unit": "MB/s", "cores": 1, "kind": "port", "seconds": t,
            "sample": f"first {len(sample) / 1e6:.1f} MB of the workload text, one Python thread "
                      "(same algorithm and speed class as the reference's OBJReader)"}


def run_obj(args):
    """OBJ ingestion: the seeded 8-copy displaced-icosphere OBJ text
    (2.6 M triangles, ~206 MB) parsed into the IndexedMesh arrays.  value:
    text MB per second of device time (CUDA events around the kernels);
    e2e: the same through parse_obj_bytes with the host text in and host
    arrays out (upload, download and the host's reading of listed lines
    inside the timed region)."""
    import workloads
    from scene.io.obj_reader import parse_obj_bytes

    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    text = workloads.obj_text()
    if args.impl == "reference":
        vals = [_obj_cpu_baseline(text, seconds_target=max(2.0, 40.0 / max(args.steps + args.warmup, 1)))
                for _ in range(args.warmup + args.steps)][args.warmup:]
        v = statistics.mean(c["value"] for c in vals)
        line = {"impl": "reference", "metric": "MB/s", "value": v, "unit": "MB/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": statistics.mean(c["seconds"] for c in vals) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64/i32",
                "data": "synthetic (seeded generator)",
                "config": {"workload": "OBJ ingestion: 8 displaced icospheres, 2.6 M triangles, "
                                       f"{len(text) / 1e6:.0f} MB of text"},
                "cpu_baseline": {k: vals[0][k] for k in ("unit", "cores", "kind", "sample")} | {"value": v},
                "e2e": {"value": v, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    import roxy_native as nat
    nat.context(0)
    for _ in range(args.warmup):
        d = parse_obj_bytes(text)
    walls, devs = [], []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            d = parse_obj_bytes(text)
            walls.append(time.perf_counter() - t0)
            devs.append(d.device_ms / 1e3)
    mb = len(text) / 1e6
    out_bytes = sum(a.nbytes for a in (d.positions, d.normals, d.uvs, d.tri_pos_idx, d.tri_normal_idx,
                                       d.tri_uv_idx, d.tri_group_idx))
    dev = statistics.mean(devs)
    peak, src = _peaks()
    alg = len(text) + out_bytes  # text read once, arrays written once
    line = {"metric": "MB/s", "value": mb / dev, "unit": "MB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64/i32", "data": "synthetic (seeded generator)",
            "config": {"workload": f"OBJ ingestion: 8 displaced icospheres, {d.triangle_count:,} triangles, "
                                   f"{mb:.0f} MB of text (larger than L2)", "triangles": d.triangle_count,
                       "vertices": int(len(d.positions))},
            "roofline": {"bound": "hbm", "kernel": "OBJ parse (line split, classify, scans, emit)",
                         "achieved": alg / dev / 1e9, "peak": peak, "unit": "GB/s", "frac": alg / dev / 1e9 / peak,
                         "peak_source": src, "traffic": None,
                         "algorithmic_bytes": alg},
            "e2e": {"value": mb / statistics.mean(walls), "unit": "MB/s", "h2d_bytes_per_step": len(text),
                    "d2h_bytes_per_step": out_bytes},
            "gpu_launches": OBJ_KERNELS_PER_PARSE * args.steps,
            "clocks": clocks.summary()}
    if not args.no_cpu:
        cb = _obj_cpu_baseline(text)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line))
    return 0


def run_serve(args):
    """Serving configuration: Poisson arrivals at swept rates.  By default
    (--serve-scenes fresh) every request arrives as a world from the
    large-mesh generator (eight seeds, 2024-2031, generated on the host
    before the sweep) and its scene is extracted and its BVH built on the
    device when it arrives, inside the request's latency; requests are
    1920x1080, 64 spp, depth 12 as in that configuration
    (--serve-sizes c2).  --serve-scenes resident reuses four resident
    scenes, --serve-sizes mixed draws 256^2-1024^2 and 1-64 spp.  The
    batched server (continuous batching, 150 GB admission budget, 1-spp
    preview first) is compared with the plain path: the same server with
    one active request at a time.  Every rate uses the same seeded request
    list (the first N of one draw)."""
    import roxy_native as nat
    import workloads
    from rendering.batch import Job
    from rendering.serving import RenderServer, poisson_run
    from rendering.taichi.extractor import build_device_scene
    from rendering.taichi.trace import make_params

    ws, rank, local = _dist()
    if rank != 0:
        return 0
    ctx = nat.context(0)
    fresh = args.serve_scenes == "fresh"
    c2 = args.serve_sizes == "c2"
    t0 = time.perf_counter()
    n_worlds = 8 if fresh else 4
    aspect = (1920, 1080) if c2 else (64, 64)
    worlds = [workloads.displaced_icosphere_scene(*aspect, seed=2024 + k) for k in range(n_worlds)]
    pool = [] if fresh else [Job(w, 64, 64, 1, 12).prepare(ctx=ctx) for w in worlds]
    gen_s = time.perf_counter() - t0
    max_req = args.max_requests or (120 if c2 else 600)
    rng = np.random.default_rng(99)
    build_ms = []

    # A request's scene is built on the server's own context while holding
    # its lock: the build waits for the step in flight, then runs alone at
    # full speed and the next step waits for it.  (Built on other contexts,
    # the build's ~100 small kernels and level read-backs interleaved with
    # the steps' long launches and each build took ~50 ms under load.)
    def fresh_request(world, W, H, spp, seed):
        def prepare():
            tb = time.perf_counter()
            with ctx.hold():
                ds = build_device_scene(world, method="lbvh", ctx=ctx)
                ds.use_lights(False)
            cam = world.active_camera
            p = make_params(W, H, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, 12, int(world._use_sky), 0,
                            1, 10.0, list(world._background_color), list(cam.position), list(cam.forward),
                            list(cam.right), list(cam.up), seed=seed)
            build_ms.append((time.perf_counter() - tb) * 1e3)
            return ds.native, p, spp, ds
        return prepare

    all_reqs = []
    for _ in range(max_req):
        k = int(rng.integers(0, n_worlds))
        if c2:
            W, H, spp = 1920, 1080, 64
        else:
            W = H = int(rng.choice([256, 512, 1024]))
            spp = int(rng.choice([1, 4, 16, 64]))
        seed = int(rng.integers(0, 1 << 30))
        if fresh:
            all_reqs.append(fresh_request(worlds[k], W, H, spp, seed))
        else:
            j = Job(worlds[k], W, H, spp, 12, scene=pool[k].scene, seed=seed).prepare(ctx=ctx)
            all_reqs.append((j.scene.native, j.params, j.spp))
    rates = [float(r) for r in args.rates.split(",")]
    rows = []
    for rate in rates:
        n = int(min(max(rate * args.duration, 20), max_req))
        reqs = all_reqs[:n]
        row = {"rate_rps": rate, "requests": n}
        # steps and waves sized to the requests: by default 32 M paths (a
        # quarter of a 1080p 64-spp request, ~9 ms) for full-HD requests,
        # 8 M for the mixed sizes; a scene build waits for the step in flight
        big = args.serve_step_paths or (1 << 25 if c2 else 1 << 23)
        for name, kw in (("batched", dict(max_active=1024, step_paths=big, wave_paths=max(big, 1 << 25))),
                         ("plain", dict(max_active=1, step_paths=1 << 40, wave_paths=max(big, 1 << 25)))):
            srv = RenderServer(hbm_budget=150e9, preview_frames=1, ctx=ctx, **kw)
            threads = args.prepare_threads if fresh else 1
            poisson_run(srv, all_reqs[-4:], rate=rate, seed=1, prepare_threads=threads)  # warm
            st0 = srv.stats()
            build_ms.clear()
            with ClockSampler(0) as clocks:
                r = poisson_run(srv, reqs, rate=rate, seed=2, prepare_threads=threads)
            st = srv.stats()
            srv.close()
            row[name] = {k: r[k] for k in ("preview_p50_ms", "preview_p99_ms", "final_p50_ms", "final_p99_ms",
                                           "throughput_rps", "prepare_p50_ms", "prepare_p99_ms")}
            row[name].update(max_active=st["max_active_seen"], max_gb=st["max_bytes_in_use"] / 1e9,
                             steps=st["steps"] - st0["steps"], busy_s=st["busy_s"] - st0["busy_s"],
                             clocks=clocks.summary())
            if build_ms:
                row[name]["scene_build_ms_p50"] = float(np.percentile(build_ms, 50))
        rows.append(row)
    top = rows[-1]
    desc = ("Poisson arrivals; each request a displaced-icosphere world (327,680 tris + 64 spheres, "
            + ("8 seeds, extracted + BVH-built on arrival" if fresh else "4 resident scenes") + "), "
            + ("1920x1080, 64 spp" if c2 else "256^2-1024^2, 1-64 spp") + ", depth 12, 150 GB budget, 1-spp preview")
    line = {"metric": "requests/s", "value": top["batched"]["throughput_rps"], "unit": "requests/s", "n_gpus": 1,
            "steps": len(rates), "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": desc, "world_generation_s": gen_s, "rates_rps": rates,
                       "prepare_threads": args.prepare_threads if fresh else 1,
                       "step_paths": args.serve_step_paths or (1 << 25 if c2 else 1 << 23),
                       "latency_from": "arrival (scene build included)" if fresh else "submission"},
            "sweep": rows,
            "speedup_vs_plain_at_top_rate": top["batched"]["throughput_rps"] / top["plain"]["throughput_rps"],
            "preview_p99_ms_at_top_rate": top["batched"]["preview_p99_ms"]}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="icosphere",
                    choices=sorted(WORKLOADS) + ["batch", "serve", "denoiser", "obj"])
    ap.add_argument("--scenes", type=int, default=64, help="scenes in the batch workload")
    ap.add_argument("--rates", default="10,50,100,200,500", help="serve workload: arrival rates (req/s)")
    ap.add_argument("--duration", type=float, default=3.0, help="serve workload: seconds of arrivals per rate")
    ap.add_argument("--max-requests", type=int, default=0,
                    help="serve workload: requests per rate at most (0: 120 for c2 sizes, 600 for mixed)")
    ap.add_argument("--serve-scenes", default="fresh", choices=["fresh", "resident"],
                    help="serve workload: build each request's scene on arrival, or reuse resident scenes")
    ap.add_argument("--serve-step-paths", type=int, default=0,
                    help="serve workload: paths per batched step (0: 2^25 for c2 sizes, 2^23 for mixed)")
    ap.add_argument("--prepare-threads", type=int, default=1,
                    help="serve workload: threads building arriving requests' scenes (fresh scenes)")
    ap.add_argument("--serve-sizes", default="c2", choices=["c2", "mixed"],
                    help="serve workload: 1920x1080 64 spp per request, or 256^2-1024^2 x 1-64 spp")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-spp", type=int, default=4096,
                    help="spp of the float64 reference render for relMSE (0: skip)")
    args = ap.parse_args()
    if args.workload == "obj":
        return run_obj(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "denoiser":
        return run_denoiser(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
