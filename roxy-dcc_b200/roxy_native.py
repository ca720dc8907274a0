"""ctypes binding of libroxy_cuda.so (the C ABI in include/roxy.h).

Every renderer, BVH and denoise entry point of this package goes through
here.  There is no CPU fallback: if the library or a CUDA device is missing,
`lib()` raises `NativeUnavailable` and the caller's operation fails.
"""
import contextlib
import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# ROXY_CUDA_LIB selects another build of the library (e.g. an installed copy)
LIB_PATH = os.environ.get("ROXY_CUDA_LIB") or os.path.join(HERE, "libroxy_cuda.so")
REPO = os.path.dirname(HERE)
SOURCES = ["rx_api.cu", "rx_bvh.cu", "rx_extract.cu", "rx_trace.cu", "rx_render.cu", "rx_denoise.cu",
           "rx_serve.cu", "rx_conv.cu", "rx_obj.cu", "rx_hostcopy.cu"]
HEADERS = ["rx_internal.cuh", "rx_runtime.h"]

RX_OK, RX_ERR_ARG, RX_ERR_CAPACITY, RX_ERR_CUDA, RX_ERR_STATE, RX_ERR_DEVICE, RX_ERR_TIMEOUT = range(7)
RX_REQ_QUEUED, RX_REQ_ACTIVE, RX_REQ_DONE, RX_REQ_FAILED = range(4)
RX_BVH_REFERENCE, RX_BVH_LBVH_SAH = 0, 1
RX_ACC_RADIANCE, RX_ACC_NORMAL, RX_ACC_ALBEDO, RX_ACC_DEPTH, RX_ACC_DISPLAY = range(5)

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


class NativeUnavailable(RuntimeError):
    """The CUDA library or a CUDA device is not available."""


class RxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class RenderParams(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("fov_tan", ctypes.c_float), ("aspect", ctypes.c_float),
        ("cam_pos", ctypes.c_float * 3), ("cam_fwd", ctypes.c_float * 3), ("cam_right", ctypes.c_float * 3),
        ("cam_up", ctypes.c_float * 3), ("max_depth", ctypes.c_int), ("use_sky", ctypes.c_int),
        ("bg", ctypes.c_float * 3), ("direct_light_mode", ctypes.c_int), ("direct_light_max_depth", ctypes.c_int),
        ("sample_clamp", ctypes.c_float), ("reference_compat", ctypes.c_int), ("seed", ctypes.c_uint32),
        ("wave_paths", ctypes.c_int), ("mis", ctypes.c_int),
    ]


class ServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_longlong), ("max_active", ctypes.c_int), ("step_paths", ctypes.c_longlong),
                ("wave_paths", ctypes.c_longlong), ("extend_block", ctypes.c_int), ("preview_frames", ctypes.c_int),
                ("pool_prewarm", ctypes.c_longlong)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("frames_done", ctypes.c_int), ("frames", ctypes.c_int),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_preview", ctypes.c_double),
                ("t_final", ctypes.c_double), ("bytes", ctypes.c_longlong)]


class ServeStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("admitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("active", ctypes.c_int), ("queued", ctypes.c_int),
                ("max_active_seen", ctypes.c_int), ("bytes_in_use", ctypes.c_longlong),
                ("max_bytes_in_use", ctypes.c_longlong), ("busy_s", ctypes.c_double), ("uptime_s", ctypes.c_double)]


class ConvDesc(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("N", "H", "W", "Cin", "Cout", "x_cstride", "x_coff", "y_cstride",
                                             "y_coff")]


class DnOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("N", ctypes.c_int), ("H", ctypes.c_int), ("W", ctypes.c_int),
                ("C", ctypes.c_int), ("a", ctypes.c_void_p), ("a_stride", ctypes.c_int), ("a_off", ctypes.c_int),
                ("b", ctypes.c_void_p), ("b_stride", ctypes.c_int), ("b_off", ctypes.c_int), ("flag", ctypes.c_int)]


RX_DN_COPY, RX_DN_RELU_MASK, RX_DN_POOL, RX_DN_POOL_BWD, RX_DN_UP, RX_DN_UP_BWD = range(6)
(RX_OBJ_SKIP, RX_OBJ_V, RX_OBJ_VN, RX_OBJ_VT, RX_OBJ_F, RX_OBJ_USEMTL, RX_OBJ_MTLLIB, RX_OBJ_O, RX_OBJ_G, RX_OBJ_S,
 RX_OBJ_OTHER) = range(11)
RX_OBJ_HOST, RX_OBJ_NONASCII = 1, 2


class DenoiseParams(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_int), ("passes", ctypes.c_int), ("sigma_color", ctypes.c_float),
        ("sigma_normal", ctypes.c_float), ("sigma_albedo", ctypes.c_float), ("sigma_depth", ctypes.c_float),
        ("amount", ctypes.c_float), ("use_normal", ctypes.c_int), ("use_albedo", ctypes.c_int),
        ("use_depth", ctypes.c_int), ("to_display", ctypes.c_int),
    ]


def nvcc_command(out=LIB_PATH):
    csrc = os.path.join(HERE, "csrc")
    return ["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
            "-fmad=false", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static", "-o", out] + \
        [os.path.join(csrc, s) for s in SOURCES]


def build(force=False):
    """Compile libroxy_cuda.so in-tree for sm_100a."""
    csrc = os.path.join(HERE, "csrc")
    deps = [os.path.join(csrc, s) for s in SOURCES + HEADERS] + [os.path.join(REPO, "include", "roxy.h")]
    if not force and os.path.exists(LIB_PATH):
        t = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB_PATH
    subprocess.run(nvcc_command(), check=True)
    return LIB_PATH


_LIB = None
_LOCK = threading.Lock()

_SIGS = {
    "rx_version": ([], ctypes.c_int),
    "rx_device_count": ([_i32p], ctypes.c_int),
    "rx_ctx_create": ([ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rx_ctx_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rx_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "rx_ctx_sync": ([ctypes.c_void_p], ctypes.c_int),
    "rx_ctx_hold": ([ctypes.c_void_p], ctypes.c_int),
    "rx_ctx_release": ([ctypes.c_void_p], ctypes.c_int),
    "rx_ctx_stream": ([ctypes.c_void_p], ctypes.c_void_p),
    "rx_scene_create": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rx_scene_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rx_scene_set_triangles": ([ctypes.c_void_p, ctypes.c_int] + [_f32p] * 6 + [_i32p], ctypes.c_int),
    "rx_scene_alloc_triangles": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_scene_put_triangles": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [_f32p] * 6 + [_i32p], ctypes.c_int),
    "rx_scene_put_indexed": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p, _i32p, ctypes.c_int,
                              _f64p, _i32p, _f64p, _f64p, _i32p, ctypes.c_int, _i32p], ctypes.c_int),
    "rx_scene_get_triangles": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [_f32p] * 6 + [_i32p], ctypes.c_int),
    "rx_scene_put_uvs": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p, _i32p], ctypes.c_int),
    "rx_scene_set_textures": ([ctypes.c_void_p, ctypes.c_int, _i32p, _i32p, _i32p, ctypes.c_void_p], ctypes.c_int),
    "rx_scene_set_material_textures": ([ctypes.c_void_p, ctypes.c_int, _i32p], ctypes.c_int),
    "rx_scene_set_materials": ([ctypes.c_void_p, ctypes.c_int, _i32p, _f32p, _f32p, _f32p, _f32p], ctypes.c_int),
    "rx_scene_set_objects": ([ctypes.c_void_p, ctypes.c_int, _i32p] + [_f32p] * 8 + [_i32p] + [_f32p] * 4,
                             ctypes.c_int),
    "rx_scene_set_lights": ([ctypes.c_void_p, ctypes.c_int, _i32p] + [_f32p] * 8 + [_i32p], ctypes.c_int),
    "rx_scene_set_light_sources": ([ctypes.c_void_p, ctypes.c_int, _i32p], ctypes.c_int),
    "rx_bvh_build": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "rx_bvh_set_reference": ([ctypes.c_void_p, ctypes.c_int, _f32p, _f32p, _i32p, _i32p, _i32p, _i32p, _i32p],
                             ctypes.c_int),
    "rx_bvh_info": ([ctypes.c_void_p] + [_i32p] * 5, ctypes.c_int),
    "rx_bvh_export_reference": ([ctypes.c_void_p, _f32p, _f32p] + [_i32p] * 5, ctypes.c_int),
    "rx_bvh_export_layout": ([ctypes.c_void_p, _f32p, _i32p], ctypes.c_int),
    "rx_trace_closest": ([ctypes.c_void_p, ctypes.c_long, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p], ctypes.c_int),
    "rx_trace_closest_device": ([ctypes.c_void_p, ctypes.c_long] + [ctypes.c_void_p] * 6, ctypes.c_int),
    "rx_trace_any": ([ctypes.c_void_p, ctypes.c_long, _f32p, _f32p, _f32p, _i32p], ctypes.c_int),
    "rx_scene_intersect": ([ctypes.c_void_p, ctypes.c_long, _f32p, _f32p, _f32p, _i32p, _i32p, _f32p, _f32p, _f32p],
                           ctypes.c_int),
    "rx_accum_create": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
                        ctypes.c_int),
    "rx_accum_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rx_accum_reset": ([ctypes.c_void_p], ctypes.c_int),
    "rx_render": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(RenderParams), ctypes.c_int], ctypes.c_int),
    "rx_accum_read": ([ctypes.c_void_p, ctypes.c_int, _f32p], ctypes.c_int),
    "rx_accum_info": ([ctypes.c_void_p, _i32p, _i32p, _i32p, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "rx_accum_denoise": ([ctypes.c_void_p, ctypes.POINTER(DenoiseParams), _f32p], ctypes.c_int),
    "rx_accum_set_timing": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_accum_set_async": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_accum_set_tail": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_accum_last_timing": ([ctypes.c_void_p, _f32p, _f32p, ctypes.c_int, _i32p], ctypes.c_int),
    "rx_accum_set_f64": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_batch_create": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rx_batch_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rx_batch_clear": ([ctypes.c_void_p], ctypes.c_int),
    "rx_batch_add": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(RenderParams), ctypes.c_int,
                      _i32p], ctypes.c_int),
    "rx_batch_set_config": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int], ctypes.c_int),
    "rx_batch_set_tail": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_batch_render": ([ctypes.c_void_p], ctypes.c_int),
    "rx_batch_last_stats": ([ctypes.c_void_p, _f32p, _i32p, _i32p], ctypes.c_int),
    "rx_accum_read_f64": ([ctypes.c_void_p, _f64p], ctypes.c_int),
    "rx_serve_create": ([ctypes.c_void_p, ctypes.POINTER(ServeConfig), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rx_serve_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rx_serve_submit": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(RenderParams), ctypes.c_int, _i32p],
                        ctypes.c_int),
    "rx_serve_info": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(RequestInfo)], ctypes.c_int),
    "rx_serve_wait": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "rx_serve_read": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _f32p], ctypes.c_int),
    "rx_serve_release": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_serve_get_stats": ([ctypes.c_void_p, ctypes.POINTER(ServeStats)], ctypes.c_int),
    "rx_scene_device_bytes": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)], ctypes.c_int),
    "rx_conv_bf16_fwd": ([ctypes.c_void_p, ctypes.POINTER(ConvDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "rx_conv_set_impl": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rx_conv_bf16_bwd_data": ([ctypes.c_void_p, ctypes.POINTER(ConvDesc)] + [ctypes.c_void_p] * 5, ctypes.c_int),
    "rx_conv_bf16_bwd_weight": ([ctypes.c_void_p, ctypes.POINTER(ConvDesc)] + [ctypes.c_void_p] * 5, ctypes.c_int),
    "rx_dn_layer": ([ctypes.c_void_p, ctypes.POINTER(DnOp), ctypes.c_void_p], ctypes.c_int),
    "rx_dn_features": ([ctypes.c_void_p, ctypes.c_longlong] + [ctypes.c_void_p] * 7, ctypes.c_int),
    "rx_dn_l1_loss": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                       ctypes.c_void_p], ctypes.c_int),
    "rx_dn_output": ([ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                      ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rx_dn_adam": ([ctypes.c_void_p, ctypes.c_longlong] + [ctypes.c_void_p] * 5 + [ctypes.c_float] * 4 +
                   [ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "rx_denoise": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p, _f32p,
                    ctypes.POINTER(DenoiseParams), _f32p], ctypes.c_int),
    "rx_denoise_noalloc": ([ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.POINTER(DenoiseParams), ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rx_obj_begin": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_void_p), _i32p,
                      _i32p], ctypes.c_int),
    "rx_obj_listed": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p], ctypes.c_int),
    "rx_obj_correct": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                       ctypes.c_int),
    "rx_obj_scan": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rx_obj_emit": ([ctypes.c_void_p] + [ctypes.c_void_p] * 8, ctypes.c_int),
    "rx_obj_device_ms": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "rx_obj_end": ([ctypes.c_void_p], ctypes.c_int),
}


def load_library(path=LIB_PATH):
    """dlopen the library and declare every exported signature (no GPU needed)."""
    if not os.path.exists(path):
        raise NativeUnavailable(f"{path} is missing; build it with __graft_entry__.build()")
    L = ctypes.CDLL(path)
    for name, (args, res) in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


def lib():
    global _LIB
    with _LOCK:
        if _LIB is None:
            _LIB = load_library()
        return _LIB


def fptr(a):
    return None if a is None else a.ctypes.data_as(_f32p)


def iptr(a):
    return None if a is None else a.ctypes.data_as(_i32p)


def f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None:
        a = a.reshape(shape)
    return a


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One device + stream.  Shared process-wide per device (see context())."""

    def __init__(self, device=0):
        L = lib()
        n = ctypes.c_int(0)
        L.rx_device_count(ctypes.byref(n))
        if n.value <= 0:
            raise NativeUnavailable("no CUDA device is visible to libroxy_cuda.so")
        h = ctypes.c_void_p()
        self._check(L.rx_ctx_create(int(device), ctypes.byref(h)), None)
        self.h = h
        self.device = device

    def _check(self, rc, handle=None):
        if rc != RX_OK:
            msg = lib().rx_last_error(handle if handle is not None else getattr(self, "h", None))
            msg = msg.decode() if msg else f"error {rc}"
            if rc == RX_ERR_ARG:
                raise ValueError(msg)
            if rc == RX_ERR_TIMEOUT:
                raise TimeoutError(msg)
            if rc == RX_ERR_CAPACITY:
                raise AssertionError(msg)
            raise RxError(rc, msg)

    def check(self, rc):
        self._check(rc, self.h)

    @property
    def stream(self):
        return lib().rx_ctx_stream(self.h)

    def sync(self):
        self.check(lib().rx_ctx_sync(self.h))

    @contextlib.contextmanager
    def hold(self):
        """Holds the context's lock for a block of calls from this thread:
        other threads' calls on the context (a serving loop's steps) wait
        until the block ends."""
        self.check(lib().rx_ctx_hold(self.h))
        try:
            yield self
        finally:
            lib().rx_ctx_release(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().rx_ctx_destroy(self.h)
            self.h = None


_CTX = {}


def context(device=0):
    if device not in _CTX:
        _CTX[device] = Context(device)
    return _CTX[device]


class NativeScene:
    """Owns an rx_scene: triangles, palette, object slots, lights and a BVH."""

    def __init__(self, ctx=None):
        self.ctx = ctx or context()
        h = ctypes.c_void_p()
        self.ctx.check(lib().rx_scene_create(self.ctx.h, ctypes.byref(h)))
        self.h = h
        self.n_tris = 0
        self.n_objects = 0
        self.n_lights = 0

    def set_triangles(self, v0, v1, v2, n0=None, n1=None, n2=None, mat_idx=None):
        v0, v1, v2 = f32(v0, (-1, 3)), f32(v1, (-1, 3)), f32(v2, (-1, 3))
        n = len(v0)
        n0 = f32(n0, (-1, 3)) if n0 is not None else np.tile(np.float32([0, 0, 1]), (n, 1))
        n1 = f32(n1, (-1, 3)) if n1 is not None else n0
        n2 = f32(n2, (-1, 3)) if n2 is not None else n0
        mat = i32(mat_idx) if mat_idx is not None else np.zeros(n, np.int32)
        if not (len(v1) == len(v2) == len(n0) == len(n1) == len(n2) == len(mat) == n):
            raise ValueError("triangle arrays must all have the same length")
        self.ctx.check(lib().rx_scene_set_triangles(self.h, n, fptr(v0), fptr(v1), fptr(v2), fptr(n0), fptr(n1),
                                                    fptr(n2), iptr(mat)))
        self.n_tris = n

    # -- piecewise extraction on the device --------------------------------------
    def alloc_triangles(self, n):
        self.ctx.check(lib().rx_scene_alloc_triangles(self.h, int(n)))
        self.n_tris = int(n)

    def put_triangles(self, offset, v0, v1, v2, n0=None, n1=None, n2=None, mat_idx=None):
        v0, v1, v2 = f32(v0, (-1, 3)), f32(v1, (-1, 3)), f32(v2, (-1, 3))
        n = len(v0)
        rows = [f32(a, (-1, 3)) if a is not None else None for a in (n0, n1, n2)]
        mat = i32(mat_idx) if mat_idx is not None else None
        if any(len(a) != n for a in [v1, v2] + [r for r in rows if r is not None]) or (mat is not None and
                                                                                        len(mat) != n):
            raise ValueError("triangle arrays must all have the same length")
        self.ctx.check(lib().rx_scene_put_triangles(self.h, int(offset), n, fptr(v0), fptr(v1), fptr(v2),
                                                    *[fptr(r) for r in rows], iptr(mat)))

    def put_indexed(self, offset, positions, tri_pos_idx, normals=None, tri_normal_idx=None, matrix=None,
                    normal_matrix=None, tri_group_idx=None, group_mat=None):
        """Rows [offset, offset + len(tri_pos_idx)) from an indexed mesh,
        transformed on the device (rx_scene_put_indexed)."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape((-1, 3))
        tri = i32(tri_pos_idx).reshape((-1, 3))
        n = len(tri)
        nrm = tn = None
        if normals is not None and tri_normal_idx is not None:
            nrm = np.ascontiguousarray(normals, dtype=np.float64).reshape((-1, 3))
            tn = i32(tri_normal_idx).reshape((-1, 3))
            if len(tn) != n:
                raise ValueError("tri_normal_idx must have one row per triangle")
        gi = None
        if tri_group_idx is not None:
            gi = i32(tri_group_idx).reshape(-1)
            if len(gi) != n:
                raise ValueError("tri_group_idx must have one entry per triangle")
        gm = i32(group_mat if group_mat is not None else [0]).reshape(-1)
        m4 = lambda m: None if m is None else np.ascontiguousarray(m, dtype=np.float64).reshape(16)  # noqa: E731
        M, NM = m4(matrix), m4(normal_matrix)
        dp = lambda a: None if a is None else a.ctypes.data_as(_f64p)  # noqa: E731
        self.ctx.check(lib().rx_scene_put_indexed(self.h, int(offset), n, len(pos), dp(pos), iptr(tri),
                                                  0 if nrm is None else len(nrm), dp(nrm), iptr(tn), dp(M), dp(NM),
                                                  iptr(gi), len(gm), iptr(gm)))

    def put_uvs(self, offset, uv0, uv1, uv2, has_uv=None):
        uv0, uv1, uv2 = (np.ascontiguousarray(a, dtype=np.float32).reshape((-1, 2)) for a in (uv0, uv1, uv2))
        n = len(uv0)
        hu = None if has_uv is None else i32(has_uv).reshape(-1)
        if len(uv1) != n or len(uv2) != n or (hu is not None and len(hu) != n):
            raise ValueError("uv arrays must all have the same length")
        self.ctx.check(lib().rx_scene_put_uvs(self.h, int(offset), n, fptr(uv0), fptr(uv1), fptr(uv2), iptr(hu)))

    def set_textures(self, images, flip_v=None):
        """images: list of (H, W, 3) uint8 arrays."""
        imgs = [np.ascontiguousarray(im, dtype=np.uint8).reshape((im.shape[0], im.shape[1], 3)) for im in images]
        n = len(imgs)
        w = np.array([im.shape[1] for im in imgs], np.int32)
        h = np.array([im.shape[0] for im in imgs], np.int32)
        fv = np.zeros(n, np.int32) if flip_v is None else i32(flip_v).reshape(n)
        texels = np.concatenate([im.reshape(-1) for im in imgs]) if n else np.zeros(0, np.uint8)
        self.ctx.check(lib().rx_scene_set_textures(self.h, n, iptr(w), iptr(h), iptr(fv),
                                                   texels.ctypes.data_as(ctypes.c_void_p) if n else None))

    def set_material_textures(self, texture_idx):
        t = i32(texture_idx).reshape(-1)
        self.ctx.check(lib().rx_scene_set_material_textures(self.h, len(t), iptr(t)))

    def get_triangles(self, offset=0, n=None):
        n = self.n_tris - offset if n is None else int(n)
        out = [np.empty((n, 3), np.float32) for _ in range(6)]
        mat = np.empty(n, np.int32)
        self.ctx.check(lib().rx_scene_get_triangles(self.h, int(offset), n, *[fptr(a) for a in out], iptr(mat)))
        return dict(zip(("v0", "v1", "v2", "n0", "n1", "n2"), out), mat_idx=mat)

    def device_bytes(self):
        n = ctypes.c_longlong()
        self.ctx.check(lib().rx_scene_device_bytes(self.h, ctypes.byref(n)))
        return n.value

    def set_materials(self, mat_type, albedo, roughness, ior, emission):
        t = i32(mat_type)
        n = len(t)
        self.ctx.check(lib().rx_scene_set_materials(self.h, n, iptr(t), fptr(f32(albedo, (-1, 3))),
                                                    fptr(f32(roughness)), fptr(f32(ior)), fptr(f32(emission))))

    def set_objects(self, slots):
        """slots: dict of arrays in the reference's _obj_* layout (len n)."""
        n = 0 if not slots else len(slots["type"])
        if n == 0:
            self.ctx.check(lib().rx_scene_set_objects(self.h, 0, *([None] * 14)))
            self.n_objects = 0
            return
        g = {k: f32(slots[k], (-1, 3)) for k in ("center", "normal", "extra", "v0", "v1", "v2", "albedo")}
        s = {k: f32(slots[k]) for k in ("radius", "offset", "roughness", "ior", "emission")}
        self.ctx.check(lib().rx_scene_set_objects(
            self.h, n, iptr(i32(slots["type"])), fptr(g["center"]), fptr(s["radius"]), fptr(g["normal"]),
            fptr(s["offset"]), fptr(g["extra"]), fptr(g["v0"]), fptr(g["v1"]), fptr(g["v2"]),
            iptr(i32(slots["mat_type"])), fptr(g["albedo"]), fptr(s["roughness"]), fptr(s["ior"]),
            fptr(s["emission"])))
        self.n_objects = n

    def set_lights(self, lights):
        n = 0 if not lights else len(lights["kind"])
        if n == 0:
            self.ctx.check(lib().rx_scene_set_lights(self.h, 0, *([None] * 10)))
            self.n_lights = 0
            return
        self.ctx.check(lib().rx_scene_set_lights(
            self.h, n, iptr(i32(lights["kind"])), fptr(f32(lights["p0"], (-1, 3))), fptr(f32(lights["p1"], (-1, 3))),
            fptr(f32(lights["p2"], (-1, 3))), fptr(f32(lights["albedo"], (-1, 3))), fptr(f32(lights["emission"])),
            fptr(f32(lights["area"])), fptr(f32(lights["pick_pdf"])), fptr(f32(lights["alias_prob"])),
            iptr(i32(lights["alias_idx"]))))
        if lights.get("source") is not None:
            self.ctx.check(lib().rx_scene_set_light_sources(self.h, n, iptr(i32(lights["source"]))))
        self.n_lights = n

    def build_bvh(self, method=RX_BVH_LBVH_SAH, max_leaf=4, spheres_in_bvh=True):
        self.ctx.check(lib().rx_bvh_build(self.h, int(method), int(max_leaf), int(bool(spheres_in_bvh))))

    def set_reference_bvh(self, node_min, node_max, left, right, start, count, order):
        n = len(left)
        self.ctx.check(lib().rx_bvh_set_reference(self.h, n, fptr(f32(node_min, (-1, 3))),
                                                  fptr(f32(node_max, (-1, 3))), iptr(i32(left)), iptr(i32(right)),
                                                  iptr(i32(start)), iptr(i32(count)), iptr(i32(order))))

    def bvh_info(self):
        v = [ctypes.c_int() for _ in range(5)]
        self.ctx.check(lib().rx_bvh_info(self.h, *[ctypes.byref(x) for x in v]))
        return dict(n_nodes=v[0].value, n_prims=v[1].value, method=v[2].value, leaf_size=v[3].value,
                    depth=v[4].value)

    def export_reference(self):
        info = self.bvh_info()
        nn = info["n_nodes"]
        out = dict(node_min=np.zeros((nn, 3), np.float32), node_max=np.zeros((nn, 3), np.float32),
                   left=np.zeros(nn, np.int32), right=np.zeros(nn, np.int32), start=np.zeros(nn, np.int32),
                   count=np.zeros(nn, np.int32), order=np.zeros(max(self.n_tris, 1), np.int32))
        self.ctx.check(lib().rx_bvh_export_reference(self.h, fptr(out["node_min"]), fptr(out["node_max"]),
                                                     iptr(out["left"]), iptr(out["right"]), iptr(out["start"]),
                                                     iptr(out["count"]), iptr(out["order"])))
        out["order"] = out["order"][: self.n_tris]
        return out

    def export_layout(self):
        info = self.bvh_info()
        nodes = np.zeros((info["n_nodes"], 16), np.float32)
        order = np.zeros(max(info["n_prims"], 1), np.int32)
        self.ctx.check(lib().rx_bvh_export_layout(self.h, fptr(nodes), iptr(order)))
        return nodes, order[: info["n_prims"]]

    def trace_closest(self, ro, rd):
        ro, rd = f32(ro, (-1, 3)), f32(rd, (-1, 3))
        n = len(ro)
        t = np.zeros(n, np.float32)
        idx = np.zeros(n, np.int32)
        u = np.zeros(n, np.float32)
        v = np.zeros(n, np.float32)
        self.ctx.check(lib().rx_trace_closest(self.h, n, fptr(ro), fptr(rd), fptr(t), iptr(idx), fptr(u), fptr(v)))
        return t, idx, u, v

    def trace_any(self, ro, rd, tmax):
        ro, rd, tmax = f32(ro, (-1, 3)), f32(rd, (-1, 3)), f32(tmax)
        n = len(ro)
        out = np.zeros(n, np.int32)
        self.ctx.check(lib().rx_trace_any(self.h, n, fptr(ro), fptr(rd), fptr(tmax), iptr(out)))
        return out

    def intersect(self, ro, rd):
        ro, rd = f32(ro, (-1, 3)), f32(rd, (-1, 3))
        n = len(ro)
        out = dict(t=np.zeros(n, np.float32), kind=np.zeros(n, np.int32), id=np.zeros(n, np.int32),
                   u=np.zeros(n, np.float32), v=np.zeros(n, np.float32), normal=np.zeros((n, 3), np.float32))
        self.ctx.check(lib().rx_scene_intersect(self.h, n, fptr(ro), fptr(rd), fptr(out["t"]), iptr(out["kind"]),
                                                iptr(out["id"]), fptr(out["u"]), fptr(out["v"]),
                                                fptr(out["normal"])))
        return out

    def close(self):
        if getattr(self, "h", None) is not None and _LIB is not None:
            _LIB.rx_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """An rx_batch: jobs (NativeScene, Accumulator, RenderParams, frames)
    rendered together as shared wavefronts in one CUDA graph."""

    def __init__(self, ctx=None):
        self.ctx = ctx or context()
        h = ctypes.c_void_p()
        self.ctx.check(lib().rx_batch_create(self.ctx.h, ctypes.byref(h)))
        self.h = h
        self._keep = []

    def add(self, scene, acc, params, frames):
        p = type(params).from_buffer_copy(params)
        job = ctypes.c_int(-1)
        self.ctx.check(lib().rx_batch_add(self.h, scene.h, acc.h, ctypes.byref(p), int(frames), ctypes.byref(job)))
        self._keep.append((scene, acc, p))
        return job.value

    def clear(self):
        self.ctx.check(lib().rx_batch_clear(self.h))
        self._keep = []

    def set_config(self, wave_paths, extend_block=128):
        self.ctx.check(lib().rx_batch_set_config(self.h, int(wave_paths), int(extend_block)))

    def set_tail(self, max_paths):
        """Wave queue length at or below which one launch runs the remaining
        bounces path by path (0: one launch pair per bounce throughout)."""
        self.ctx.check(lib().rx_batch_set_tail(self.h, int(max_paths)))

    def render(self):
        self.ctx.check(lib().rx_batch_render(self.h))

    def last_stats(self):
        ms = ctypes.c_float()
        waves = ctypes.c_int()
        launches = ctypes.c_int()
        self.ctx.check(lib().rx_batch_last_stats(self.h, ctypes.byref(ms), ctypes.byref(waves), ctypes.byref(launches)))
        return dict(ms=ms.value, waves=waves.value, launches=launches.value)

    def close(self):
        if getattr(self, "h", None) is not None and _LIB is not None:
            _LIB.rx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Accumulator:
    """rx_accum: progressive running means and wavefront buffers for W x H."""

    def __init__(self, width, height, ctx=None):
        self.ctx = ctx or context()
        h = ctypes.c_void_p()
        self.ctx.check(lib().rx_accum_create(self.ctx.h, int(width), int(height), ctypes.byref(h)))
        self.h = h
        self.width, self.height = int(width), int(height)

    def reset(self):
        self.ctx.check(lib().rx_accum_reset(self.h))

    def render(self, scene, params, frames):
        self.ctx.check(lib().rx_render(scene.h, self.h, ctypes.byref(params), int(frames)))

    def read(self, which, out=None):
        """One accumulator plane as float32 (H, W) or (H, W, 3); with `out`
        (C-contiguous float32 of that shape, e.g. an Image's pixels) the
        device copy lands in it directly, with no new host array."""
        shape = (self.height, self.width) if which == RX_ACC_DEPTH else (self.height, self.width, 3)
        if out is None:
            out = np.empty(shape, np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"read: out must be a C-contiguous float32 array of shape {shape}")
        self.ctx.check(lib().rx_accum_read(self.h, int(which), fptr(out)))
        return out

    def info(self):
        w, h, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        r = ctypes.c_longlong()
        self.ctx.check(lib().rx_accum_info(self.h, ctypes.byref(w), ctypes.byref(h), ctypes.byref(f),
                                           ctypes.byref(r)))
        return dict(width=w.value, height=h.value, frames=f.value, rays=r.value)

    def denoise(self, params, out=True):
        res = np.zeros((self.height, self.width, 3), np.float32) if out else None
        self.ctx.check(lib().rx_accum_denoise(self.h, ctypes.byref(params), fptr(res)))
        return res

    def set_timing(self, on):
        self.ctx.check(lib().rx_accum_set_timing(self.h, int(bool(on))))

    def set_async(self, on):
        """reset()/render() return once queued; errors surface at ctx.sync()."""
        self.ctx.check(lib().rx_accum_set_async(self.h, int(bool(on))))

    def set_tail(self, max_paths):
        """Queue length at or below which one launch runs a wave's remaining
        bounces path by path (0: one launch pair per bounce throughout)."""
        self.ctx.check(lib().rx_accum_set_tail(self.h, int(max_paths)))

    def last_timing(self):
        tot = ctypes.c_float()
        ks = (ctypes.c_float * 5)()
        nl = ctypes.c_int()
        self.ctx.check(lib().rx_accum_last_timing(self.h, ctypes.byref(tot), ks, 5, ctypes.byref(nl)))
        return dict(total_ms=tot.value, extend_ms=ks[0], shade_ms=ks[1], connect_ms=ks[2], other_ms=ks[3],
                    accumulate_ms=ks[4], launches=nl.value)

    def set_f64(self, on):
        """Keep float64 sums of the clamped sample radiance (reset first)."""
        self.ctx.check(lib().rx_accum_set_f64(self.h, int(bool(on))))

    def read_f64(self):
        out = np.zeros((self.height, self.width, 3), np.float64)
        self.ctx.check(lib().rx_accum_read_f64(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def close(self):
        if getattr(self, "h", None) is not None and _LIB is not None:
            _LIB.rx_accum_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def denoise(color, normal=None, albedo=None, depth=None, radius=1, sigma_color=0.08, amount=1.0,
            sigma_normal=0.35, sigma_albedo=0.20, sigma_depth=1.0, passes=1, to_display=False, ctx=None):
    """edge_aware_denoise / a-trous on host arrays through rx_denoise."""
    ctx = ctx or context()
    c = f32(color)
    H, W = c.shape[:2]
    p = DenoiseParams(int(radius), int(passes), float(sigma_color), float(sigma_normal), float(sigma_albedo),
                      float(sigma_depth), float(amount), 0, 0, 0, int(bool(to_display)))
    out = np.zeros((H, W, 3), np.float32)
    nn = f32(normal) if normal is not None else None
    aa = f32(albedo) if albedo is not None else None
    dd = f32(depth).reshape(H, W) if depth is not None else None
    ctx.check(lib().rx_denoise(ctx.h, H, W, fptr(c), fptr(nn), fptr(aa), fptr(dd), ctypes.byref(p), fptr(out)))
    return out
