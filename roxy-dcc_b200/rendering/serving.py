"""Render serving with continuous batching (rx_serve_*).

A RenderServer owns a native serving loop on its own host thread: requests
(a resident scene, render parameters, a frame count) are admitted as active
slots and the device-memory budget allow, each gets a preview in the next
step and is then refined within a per-step path budget, and every step
traces all admitted requests together as one batch of wavefronts.  Scenes
and BVHs stay resident; each request's accumulator lives until release().

poisson_run() drives a server with Poisson arrivals and reports latency to
the first preview and to the final image (p50 / p99) beside throughput.
"""
import ctypes
import time

import numpy as np

import roxy_native as nat

STATE_NAMES = {nat.RX_REQ_QUEUED: "queued", nat.RX_REQ_ACTIVE: "active", nat.RX_REQ_DONE: "done",
               nat.RX_REQ_FAILED: "failed"}


class RenderServer:
    def __init__(self, hbm_budget=150e9, max_active=256, step_paths=1 << 25, wave_paths=1 << 25, extend_block=128,
                 preview_frames=1, pool_prewarm=None, ctx=None):
        self.ctx = ctx or nat.context()
        if pool_prewarm is None:
            pool_prewarm = min(hbm_budget / 8, 16e9)
        cfg = nat.ServeConfig(int(hbm_budget), int(max_active), int(step_paths), int(wave_paths), int(extend_block),
                              int(preview_frames), int(pool_prewarm))
        h = ctypes.c_void_p()
        self.ctx.check(nat.lib().rx_serve_create(self.ctx.h, ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self._meta = {}

    def submit(self, scene, params, frames):
        """Queue a request; returns its id.  `scene`: NativeScene (kept
        alive by the server object until release)."""
        rid = ctypes.c_int(-1)
        p = type(params).from_buffer_copy(params)
        self.ctx.check(nat.lib().rx_serve_submit(self.h, scene.h, ctypes.byref(p), int(frames), ctypes.byref(rid)))
        self._meta[rid.value] = (scene, p.width, p.height)
        return rid.value

    def info(self, rid):
        out = nat.RequestInfo()
        self.ctx.check(nat.lib().rx_serve_info(self.h, int(rid), ctypes.byref(out)))
        return {"state": STATE_NAMES[out.state], "frames_done": out.frames_done, "frames": out.frames,
                "t_submit": out.t_submit, "t_admit": out.t_admit, "t_preview": out.t_preview, "t_final": out.t_final,
                "bytes": out.bytes}

    def wait(self, rid, final=True, timeout=60.0):
        self.ctx.check(nat.lib().rx_serve_wait(self.h, int(rid), int(bool(final)), float(timeout)))

    def read(self, rid, which=nat.RX_ACC_DISPLAY):
        _, w, h = self._meta[rid]
        shape = (h, w) if which == nat.RX_ACC_DEPTH else (h, w, 3)
        out = np.zeros(shape, np.float32)
        self.ctx.check(nat.lib().rx_serve_read(self.h, int(rid), int(which), nat.fptr(out)))
        return out

    def release(self, rid):
        self.ctx.check(nat.lib().rx_serve_release(self.h, int(rid)))
        self._meta.pop(rid, None)

    def stats(self):
        s = nat.ServeStats()
        self.ctx.check(nat.lib().rx_serve_get_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in nat.ServeStats._fields_}

    def close(self):
        if getattr(self, "h", None) is not None and nat._LIB is not None:
            nat._LIB.rx_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else float("nan")


def poisson_run(server, requests, rate, seed=0, read_final=False, timeout=300.0, prepare_threads=1):
    """Submit `requests` with exponential inter-arrival times of mean
    1/rate.  A request is (NativeScene, RenderParams, frames), or a callable
    that returns one: it runs when the request arrives (building the
    request's scene, say), and the time it takes counts toward the
    request's latencies.  A second thread plays the client that waits for
    each final image, reads it if asked and releases the request as soon as
    it is done, while arrivals continue.  With prepare_threads > 1 callable
    requests are prepared and submitted by that many worker threads, so one
    slow preparation does not hold back the arrivals behind it.  Returns
    latency and throughput figures (latencies from arrival)."""
    import queue
    import threading
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(requests))
    ids = queue.Queue()
    infos, errors = [], []
    prep_s = {}
    keep = {}

    def collect():
        for _ in range(len(requests)):
            rid = ids.get()
            if rid is None:
                return
            try:
                server.wait(rid, final=True, timeout=timeout)
                info = server.info(rid)
                info["prep_s"] = prep_s.get(rid, 0.0)
                infos.append(info)
                if read_final:
                    server.read(rid)
                server.release(rid)
                keep.pop(rid, None)
            except Exception as e:  # re-raised after the run
                errors.append(e)

    th = threading.Thread(target=collect, daemon=True)
    th.start()
    lock = threading.Lock()

    def arrive(req, t_arrival):
        made = req() if callable(req) else req
        scene, params, frames = made[:3]
        # a request's latency runs from its arrival: the time spent behind
        # earlier arrivals' preparation counts too
        prep = time.perf_counter() - t_arrival
        rid = server.submit(scene, params, frames)
        with lock:
            prep_s[rid] = prep
            keep[rid] = made
        ids.put(rid)

    pool = None
    if prepare_threads > 1:
        from concurrent.futures import ThreadPoolExecutor
        pool = ThreadPoolExecutor(prepare_threads)
    futures = []
    t_start = time.perf_counter()
    t_next = t_start
    try:
        for req, gap in zip(requests, gaps):
            t_next += gap
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            if pool is not None and callable(req):
                futures.append(pool.submit(arrive, req, t_next))
            else:
                arrive(req, t_next)
        for f in futures:
            f.result()
    except Exception:
        ids.put(None)
        th.join()
        raise
    finally:
        if pool is not None:
            pool.shutdown(wait=True)
    th.join()
    if errors:
        raise errors[0]
    t_end = time.perf_counter()
    prev = [i["t_preview"] - i["t_submit"] + i["prep_s"] for i in infos]
    fin = [i["t_final"] - i["t_submit"] + i["prep_s"] for i in infos]
    prep = [i["prep_s"] for i in infos]
    first = min(i["t_submit"] for i in infos)
    last = max(i["t_final"] for i in infos)
    return {"requests": len(infos), "rate": rate, "preview_p50_ms": 1e3 * percentile(prev, 50),
            "preview_p99_ms": 1e3 * percentile(prev, 99), "final_p50_ms": 1e3 * percentile(fin, 50),
            "final_p99_ms": 1e3 * percentile(fin, 99), "throughput_rps": len(infos) / max(last - first, 1e-9),
            "prepare_p50_ms": 1e3 * percentile(prep, 50), "prepare_p99_ms": 1e3 * percentile(prep, 99),
            "wall_s": t_end - t_start}
