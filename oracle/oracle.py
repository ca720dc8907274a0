"""ORACLE — test infrastructure only.

Python face of the CPU restatement of roxy-dcc's path-tracing hot path:

* `liboracle.so` (oracle.cpp): traversal, primitives, the trace loop and the
  Morton BVH build, in IEEE float32 without FMA contraction;
* `edge_aware_denoise` below: a numpy restatement of
  rendering/denoise.py:23-104 (guided bilateral filter) with the same float32
  operation order.

Only the tests, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg use
this module, and only as the checker / the timed CPU baseline.  The product
(the CUDA library and its Python host code) never imports it.

Parity pins: tests/test_oracle_golden.py checks every function here against
the golden vectors that tests/golden/make_golden.py produced by executing the
reference's own source.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int)
_u32p = ctypes.POINTER(ctypes.c_uint32)


class OrcScene(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int), ("node_min", _f32p), ("node_max", _f32p),
        ("node_left", _i32p), ("node_right", _i32p), ("node_tri_start", _i32p), ("node_tri_count", _i32p),
        ("n_tris", ctypes.c_int), ("v0", _f32p), ("v1", _f32p), ("v2", _f32p),
        ("n0", _f32p), ("n1", _f32p), ("n2", _f32p), ("tri_mat", _i32p),
        ("n_mats", ctypes.c_int), ("mat_type", _i32p), ("mat_albedo", _f32p), ("mat_roughness", _f32p),
        ("mat_ior", _f32p), ("mat_emission", _f32p),
        ("n_objects", ctypes.c_int), ("obj_type", _i32p), ("obj_center", _f32p), ("obj_radius", _f32p),
        ("obj_normal", _f32p), ("obj_offset", _f32p), ("obj_extra", _f32p),
        ("obj_v0", _f32p), ("obj_v1", _f32p), ("obj_v2", _f32p),
        ("obj_mat_type", _i32p), ("obj_albedo", _f32p), ("obj_roughness", _f32p),
        ("obj_ior", _f32p), ("obj_emission", _f32p),
        ("n_lights", ctypes.c_int), ("light_kind", _i32p), ("light_p0", _f32p), ("light_p1", _f32p),
        ("light_p2", _f32p), ("light_albedo", _f32p), ("light_emission", _f32p), ("light_area", _f32p),
        ("light_pick_pdf", _f32p), ("alias_prob", _f32p), ("alias_idx", _i32p), ("light_obj", _i32p),
        ("uv0", _f32p), ("uv1", _f32p), ("uv2", _f32p), ("has_uv", _i32p), ("mat_texture", _i32p),
        ("n_tex", ctypes.c_int), ("tex_w", _i32p), ("tex_h", _i32p), ("tex_flip", _i32p),
        ("tex_off", ctypes.POINTER(ctypes.c_longlong)), ("texels", ctypes.c_void_p),
    ]


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("fov_tan", ctypes.c_float),
        ("aspect", ctypes.c_float), ("cam_pos", ctypes.c_float * 3), ("cam_fwd", ctypes.c_float * 3),
        ("cam_right", ctypes.c_float * 3), ("cam_up", ctypes.c_float * 3), ("max_depth", ctypes.c_int),
        ("use_sky", ctypes.c_int), ("bg", ctypes.c_float * 3), ("direct_light_mode", ctypes.c_int),
        ("direct_light_max_depth", ctypes.c_int), ("sample_clamp", ctypes.c_float),
        ("reference_compat", ctypes.c_int), ("seed", ctypes.c_uint32),
    ]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(os.path.join(HERE, "oracle.cpp")):
            build()
        L = ctypes.CDLL(path)
        L.orc_render.restype = ctypes.c_long
        L.orc_render_samples.restype = ctypes.c_long
        L.orc_bvh_build_morton.restype = ctypes.c_int
        L.orc_trace_scripted.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a, t=_f32p):
    return a.ctypes.data_as(t) if a is not None else None


def _f(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Scene:
    """Owns the numpy arrays behind one OrcScene (reference flat layout)."""

    def __init__(self, *, node_min=None, node_max=None, left=None, right=None, start=None, count=None,
                 v0=None, v1=None, v2=None, n0=None, n1=None, n2=None, tri_mat=None,
                 mat_type=None, mat_albedo=None, mat_roughness=None, mat_ior=None, mat_emission=None,
                 objects=None, lights=None, uv0=None, uv1=None, uv2=None, has_uv=None, mat_texture=None,
                 textures=None, tex_flip=None):
        keep = {}
        s = OrcScene()

        def F(name, a):
            if a is None:
                return None
            a = _f(a)
            keep[name] = a
            return _p(a)

        def I(name, a):
            if a is None:
                return None
            a = _i(a)
            keep[name] = a
            return _p(a, _i32p)

        n_nodes = 0 if left is None else len(left)
        s.n_nodes = n_nodes
        s.node_min, s.node_max = F("nmin", node_min), F("nmax", node_max)
        s.node_left, s.node_right = I("l", left), I("r", right)
        s.node_tri_start, s.node_tri_count = I("s", start), I("c", count)
        s.n_tris = 0 if v0 is None else len(v0)
        s.v0, s.v1, s.v2 = F("v0", v0), F("v1", v1), F("v2", v2)
        if v0 is not None and n0 is None:
            z = np.tile(np.float32([0, 0, 1]), (len(v0), 1))
            n0 = n1 = n2 = z
        s.n0, s.n1, s.n2 = F("n0", n0), F("n1", n1), F("n2", n2)
        if v0 is not None and tri_mat is None:
            tri_mat = np.zeros(len(v0), np.int32)
        s.tri_mat = I("tm", tri_mat)
        if mat_type is None:
            mat_type = np.zeros(1, np.int32)
            mat_albedo = np.full((1, 3), 0.8, np.float32)
            mat_roughness = np.zeros(1, np.float32)
            mat_ior = np.ones(1, np.float32)
            mat_emission = np.zeros(1, np.float32)
        s.n_mats = len(mat_type)
        s.mat_type, s.mat_albedo = I("mt", mat_type), F("ma", mat_albedo)
        s.mat_roughness, s.mat_ior, s.mat_emission = F("mr", mat_roughness), F("mi", mat_ior), F("me", mat_emission)
        o = objects or {}
        s.n_objects = 0 if not o else len(o["type"])
        s.obj_type = I("ot", o.get("type"))
        s.obj_center, s.obj_radius = F("oc", o.get("center")), F("orad", o.get("radius"))
        s.obj_normal, s.obj_offset = F("on", o.get("normal")), F("oo", o.get("offset"))
        s.obj_extra = F("oe", o.get("extra"))
        s.obj_v0, s.obj_v1, s.obj_v2 = F("ov0", o.get("v0")), F("ov1", o.get("v1")), F("ov2", o.get("v2"))
        s.obj_mat_type = I("omt", o.get("mat_type"))
        s.obj_albedo, s.obj_roughness = F("oa", o.get("albedo")), F("ork", o.get("roughness"))
        s.obj_ior, s.obj_emission = F("oi", o.get("ior")), F("oem", o.get("emission"))
        L = lights or {}
        s.n_lights = 0 if not L else len(L["kind"])
        s.light_kind = I("lk", L.get("kind"))
        s.light_p0, s.light_p1, s.light_p2 = F("lp0", L.get("p0")), F("lp1", L.get("p1")), F("lp2", L.get("p2"))
        s.light_albedo, s.light_emission = F("la", L.get("albedo")), F("le", L.get("emission"))
        s.light_area, s.light_pick_pdf = F("lar", L.get("area")), F("lpp", L.get("pick_pdf"))
        s.alias_prob, s.alias_idx = F("lap", L.get("alias_prob")), I("lai", L.get("alias_idx"))
        s.light_obj = I("lo", L.get("obj"))
        # textures: uv rows in BVH order, texture index per material, list of
        # (H, W, 3) uint8 images
        s.uv0, s.uv1, s.uv2 = F("uv0", uv0), F("uv1", uv1), F("uv2", uv2)
        s.has_uv, s.mat_texture = I("huv", has_uv), I("mtex", mat_texture)
        imgs = [np.ascontiguousarray(im, dtype=np.uint8) for im in (textures or [])]
        s.n_tex = len(imgs)
        if imgs:
            s.tex_w = I("tw", [im.shape[1] for im in imgs])
            s.tex_h = I("th", [im.shape[0] for im in imgs])
            s.tex_flip = I("tf", tex_flip if tex_flip is not None else [0] * len(imgs))
            off = np.cumsum([0] + [im.size for im in imgs[:-1]]).astype(np.int64)
            keep["toff"] = off
            s.tex_off = off.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
            tx = np.concatenate([im.reshape(-1) for im in imgs])
            keep["texels"] = tx
            s.texels = tx.ctypes.data_as(ctypes.c_void_p)
        self._keep = keep
        self.s = s

    def ptr(self):
        return ctypes.byref(self.s)


def make_params(width, height, fov_tan, aspect, cam_pos, cam_fwd, cam_right, cam_up, max_depth,
                use_sky, bg, direct_light_mode=0, direct_light_max_depth=1, sample_clamp=10.0,
                reference_compat=0, seed=0):
    p = OrcParams()
    p.width, p.height, p.fov_tan, p.aspect = width, height, fov_tan, aspect
    for name, v in (("cam_pos", cam_pos), ("cam_fwd", cam_fwd), ("cam_right", cam_right),
                    ("cam_up", cam_up), ("bg", bg)):
        arr = getattr(p, name)
        for k in range(3):
            arr[k] = float(v[k])
    p.max_depth, p.use_sky = max_depth, int(use_sky)
    p.direct_light_mode, p.direct_light_max_depth = direct_light_mode, direct_light_max_depth
    p.sample_clamp, p.reference_compat, p.seed = sample_clamp, int(reference_compat), seed
    return p


# ---------------------------------------------------------------------------
# thin wrappers
# ---------------------------------------------------------------------------
def bvh_build_morton(v0, v1, v2, leaf_size=8):
    """Morton build restating GPUBVHBuilder (bvh_builder.py:412-478)."""
    v0, v1, v2 = _f(v0), _f(v1), _f(v2)
    n = len(v0)
    cap = max(2 * n - 1, 1)
    nmin = np.zeros((cap, 3), np.float32)
    nmax = np.zeros((cap, 3), np.float32)
    left = np.zeros(cap, np.int32)
    right = np.zeros(cap, np.int32)
    start = np.zeros(cap, np.int32)
    count = np.zeros(cap, np.int32)
    order = np.zeros(max(n, 1), np.int32)
    nn = lib().orc_bvh_build_morton(n, _p(v0), _p(v1), _p(v2), int(leaf_size), _p(nmin), _p(nmax),
                                    _p(left, _i32p), _p(right, _i32p), _p(start, _i32p), _p(count, _i32p),
                                    _p(order, _i32p))
    return dict(node_min=nmin[:nn], node_max=nmax[:nn], left=left[:nn], right=right[:nn],
                start=start[:nn], count=count[:nn], order=order[:n])


def bvh_intersect(scene, ro, rd):
    ro, rd = _f(ro), _f(rd)
    n = len(ro)
    t = np.zeros(n, np.float32)
    idx = np.zeros(n, np.int32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    lib().orc_bvh_intersect(scene.ptr(), ctypes.c_long(n), _p(ro), _p(rd), _p(t), _p(idx, _i32p), _p(u), _p(v))
    return t, idx, u, v


def bvh_occluded(scene, ro, rd, max_t):
    ro, rd, max_t = _f(ro), _f(rd), _f(max_t)
    n = len(ro)
    out = np.zeros(n, np.int32)
    lib().orc_bvh_occluded(scene.ptr(), ctypes.c_long(n), _p(ro), _p(rd), _p(max_t), _p(out, _i32p))
    return out


def scene_intersect(scene, ro, rd):
    ro, rd = _f(ro), _f(rd)
    n = len(ro)
    t = np.zeros(n, np.float32)
    idx = np.zeros(n, np.int32)
    isb = np.zeros(n, np.int32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    nrm = np.zeros((n, 3), np.float32)
    lib().orc_scene_intersect(scene.ptr(), ctypes.c_long(n), _p(ro), _p(rd), _p(t), _p(idx, _i32p),
                              _p(isb, _i32p), _p(u), _p(v), _p(nrm))
    return dict(t=t, idx=idx, is_bvh=isb, u=u, v=v, normal=nrm)


def tri_intersect(ro, rd, v0, v1, v2):
    ro, rd, v0, v1, v2 = (_f(a) for a in (ro, rd, v0, v1, v2))
    n = len(ro)
    t = np.zeros(n, np.float32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    lib().orc_tri_intersect(ctypes.c_long(n), _p(ro), _p(rd), _p(v0), _p(v1), _p(v2), _p(t), _p(u), _p(v))
    return t, u, v


def trace_scripted(scene, params, ro, rd, stream):
    ro, rd, stream = _f(ro), _f(rd), _f(stream)
    color = np.zeros(3, np.float32)
    nrm = np.zeros(3, np.float32)
    alb = np.zeros(3, np.float32)
    dep = np.zeros(1, np.float32)
    rays = np.zeros(1, np.int64)
    used = lib().orc_trace_scripted(scene.ptr(), ctypes.byref(params), _p(ro), _p(rd), _p(stream),
                                    len(stream), _p(color), _p(nrm), _p(alb), _p(dep),
                                    rays.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
    return dict(color=color, normal=nrm, albedo=alb, depth=float(dep[0]), consumed=used, rays=int(rays[0]))


def sample_texture(scene, tex_idx, uv):
    """_sample_texture (trace.py:96-126) at each uv row -> (n, 3)."""
    uv = _f(uv).reshape((-1, 2))
    out = np.zeros((len(uv), 3), np.float32)
    lib().orc_sample_texture(scene.ptr(), int(tex_idx), len(uv), _p(uv), _p(out))
    return out


def bvh_albedo(scene, tri, mat, u, v, base):
    """_bvh_albedo (trace.py:129-136) per (BVH-order triangle, material,
    barycentrics, base albedo) -> (n, 3)."""
    tri, mat = _i(tri), _i(mat)
    u, v, base = _f(u), _f(v), _f(base).reshape((-1, 3))
    out = np.zeros((len(tri), 3), np.float32)
    lib().orc_bvh_albedo(scene.ptr(), len(tri), _p(tri, _i32p), _p(mat, _i32p), _p(u), _p(v), _p(base), _p(out))
    return out


def render(scene, params, frames, rows=None, n_threads=0):
    """Progressive render (running means, trace.py:262-283). Returns dict of buffers."""
    W, H = params.width, params.height
    acc = np.zeros((H, W, 3), np.float32)
    accn = np.zeros((H, W, 3), np.float32)
    acca = np.zeros((H, W, 3), np.float32)
    accd = np.zeros((H, W), np.float32)
    pix = np.zeros((H, W, 3), np.float32)
    y0, y1 = rows if rows is not None else (0, H)
    rays = lib().orc_render(scene.ptr(), ctypes.byref(params), 0, int(frames), int(y0), int(y1), _p(acc), _p(accn),
                            _p(acca), _p(accd), _p(pix), int(n_threads))
    return dict(radiance=acc, normal=accn, albedo=acca, depth=accd, pixels=pix, rays=int(rays))


def render_samples(scene, params, frame0, frame1, n_threads=0):
    W, H = params.width, params.height
    out = np.zeros((frame1 - frame0, H, W, 3), np.float32)
    rays = lib().orc_render_samples(scene.ptr(), ctypes.byref(params), int(frame0), int(frame1), _p(out),
                                    int(n_threads))
    return out, int(rays)


def philox(ctr, k0, k1):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox(c.ctypes.data_as(_u32p), ctypes.c_uint32(k0), ctypes.c_uint32(k1), out.ctypes.data_as(_u32p))
    return out


# ---------------------------------------------------------------------------
# numpy restatement of rendering/denoise.py:23-108
# ---------------------------------------------------------------------------
def _guide(name, guide, shape, channels):
    if guide is None:
        return None
    arr = np.asarray(guide, dtype=np.float32)
    if arr.shape[:2] != shape:
        raise ValueError(f"{name} guide must match pixel height and width")
    if arr.ndim == 2:
        arr = arr[:, :, None]
    elif arr.ndim != 3:
        raise ValueError(f"{name} guide must be a 2D or 3D array")
    if arr.shape[2] != channels:
        raise ValueError(f"{name} guide must have {channels} channel(s)")
    return arr


def edge_aware_denoise(linear_pixels, radius=1, sigma_color=0.08, amount=1.0, *, normal=None, albedo=None,
                       depth=None, sigma_normal=0.35, sigma_albedo=0.20, sigma_depth=1.0):
    """Guided bilateral filter, same float32 op order as denoise.py:23-104."""
    if radius <= 0 or amount <= 0.0:
        return linear_pixels
    src = np.asarray(linear_pixels, dtype=np.float32)
    r = int(radius)
    H, W = src.shape[:2]
    two_s2 = np.float32(2.0 * max(float(sigma_color) ** 2, 1e-8))
    amount = min(max(float(amount), 0.0), 1.0)
    pad = np.pad(src, ((r, r), (r, r), (0, 0)), mode="reflect")
    center = pad[r:r + H, r:r + W]
    guides = []
    for g, sg, name, ch in ((normal, sigma_normal, "normal", 3), (albedo, sigma_albedo, "albedo", 3),
                            (depth, sigma_depth, "depth", 1)):
        g = _guide(name, g, (H, W), ch)
        if g is None:
            continue
        gp = np.pad(g, ((r, r), (r, r), (0, 0)), mode="reflect")
        guides.append((gp, gp[r:r + H, r:r + W], np.float32(2.0 * max(float(sg) ** 2, 1e-8))))
    acc = np.zeros_like(src)
    wsum = np.zeros((H, W), np.float32)
    for dy in range(-r, r + 1):
        for dx in range(-r, r + 1):
            nb = pad[r + dy:r + dy + H, r + dx:r + dx + W]
            d = nb - center
            d2 = np.sum(d * d, axis=2)
            w = np.float32(1.0 / (1.0 + dx * dx + dy * dy)) * np.exp(-d2 / two_s2)
            for gp, gc, gs2 in guides:
                gd = gp[r + dy:r + dy + H, r + dx:r + dx + W] - gc
                w = w * np.exp(-np.sum(gd * gd, axis=2) / gs2)
            acc += nb * w[:, :, None]
            wsum += w
    filt = acc / np.maximum(wsum[:, :, None], np.float32(1e-8))
    return src * np.float32(1.0 - amount) + filt * np.float32(amount)


def linear_to_display(x):
    return np.sqrt(np.minimum(np.maximum(x, 0.0), 1.0)).astype(np.float32)
