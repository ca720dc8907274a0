"""Learned denoiser: a 3-level convolutional encoder-decoder trained on
low-spp / high-spp pairs that the renderer produces.

Input (16 channels, NHWC bf16): log1p of the noisy radiance, first-hit
albedo, normal and depth / (1 + depth), zero-padded from 10 channels.
Network: 3x3 convolutions with ReLU,

    enc 16->32->32 | pool | 32->64->64 | pool | 64->128->128
    dec up, concat skip (128+64) -> 64 -> 64 | up, concat (64+32) -> 32 -> 32
    head 32 -> 16 (3 used)

whose output is added to log1p(noisy radiance); the image is
expm1(that).  Every layer runs in libroxy_cuda.so: BF16 tensor-core
convolutions with FP32 accumulation (rx_conv_bf16_*), element-wise layers
(rx_dn_layer), L1 loss in log1p space and Adam on FP32 master weights
(rx_dn_*).  torch provides device memory and the stream only.

The edge-aware a-trous filter (rendering/denoise.py) remains the fallback;
evaluate() reports both against a high-spp float64 reference.
"""
import ctypes
import math

import numpy as np

import roxy_native as nat

LAYERS = [  # name, input channels, output channels, relu
    ("e1a", 16, 32, 1), ("e1b", 32, 32, 1),
    ("e2a", 32, 64, 1), ("e2b", 64, 64, 1),
    ("e3a", 64, 128, 1), ("e3b", 128, 128, 1),
    ("d2a", 192, 64, 1), ("d2b", 64, 64, 1),
    ("d1a", 96, 32, 1), ("d1b", 32, 32, 1),
    ("head", 32, 16, 0),
]
REAL_IN = {"e1a": 10, "head": 32}


def _torch():
    import torch
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def macs_per_pixel():
    """Multiply-adds per full-resolution pixel of one forward pass."""
    scale = {"e1": 1, "e2": 0.25, "e3": 1 / 16, "d2": 0.25, "d1": 1, "he": 1}
    return sum(9 * cin * cout * scale[name[:2]] for name, cin, cout, _ in LAYERS)


class Denoiser:
    """Weights, Adam state and activation buffers of the network."""

    def __init__(self, ctx=None, seed=0, weights=None):
        torch = _torch()
        self.ctx = ctx or nat.context()
        self.dev = torch.device("cuda", self.ctx.device)
        self.w32, self.b32, self.w16, self.dw, self.db = {}, {}, {}, {}, {}
        self.mw, self.vw, self.mb, self.vb = {}, {}, {}, {}
        rng = np.random.default_rng(seed)
        for name, cin, cout, _ in LAYERS:
            fan = 9 * REAL_IN.get(name, cin)
            w = rng.normal(0.0, math.sqrt(2.0 / fan), size=(cout, 9, cin)).astype(np.float32)
            if name == "e1a":
                w[:, :, 10:] = 0.0
            if name == "head":
                w[3:] = 0.0
                w *= 0.1
            self.w32[name] = torch.from_numpy(w).to(self.dev)
            self.b32[name] = torch.zeros(cout, dtype=torch.float32, device=self.dev)
        if weights is not None:
            self.load(weights)
        for name, cin, cout, _ in LAYERS:
            self.w16[name] = self.w32[name].to(torch.bfloat16)
            for d, shape in ((self.dw, (cout, 9, cin)), (self.mw, (cout, 9, cin)), (self.vw, (cout, 9, cin)),
                             (self.db, (cout,)), (self.mb, (cout,)), (self.vb, (cout,))):
                d[name] = torch.zeros(shape, dtype=torch.float32, device=self.dev)
        self.step = 0
        self._bufs = {}
        self.rot = torch.empty(max(c * 9 * k for _, k, c, _ in LAYERS), dtype=torch.bfloat16, device=self.dev)
        self.loss_acc = torch.zeros(1, dtype=torch.float32, device=self.dev)

    # -- parameters ------------------------------------------------------------
    def state(self):
        out = {}
        for name, _, _, _ in LAYERS:
            out[f"{name}.w"] = self.w32[name].cpu().numpy()
            out[f"{name}.b"] = self.b32[name].cpu().numpy()
        return out

    def save(self, path):
        np.savez_compressed(path, **self.state())

    def load(self, src):
        torch = _torch()
        d = np.load(src) if isinstance(src, str) else src
        for name, cin, cout, _ in LAYERS:
            w = np.asarray(d[f"{name}.w"], np.float32).reshape(cout, 9, cin)
            self.w32[name] = torch.from_numpy(w.copy()).to(self.dev)
            self.b32[name] = torch.from_numpy(np.asarray(d[f"{name}.b"], np.float32).copy()).to(self.dev)
            if name in self.w16:
                self.w16[name] = self.w32[name].to(torch.bfloat16)

    # -- buffers ------------------------------------------------------------------
    def buffers(self, N, H, W, train):
        key = (N, H, W, train)
        if key in self._bufs:
            return self._bufs[key]
        torch = _torch()
        if H % 4 or W % 4:
            raise ValueError("image height and width must be multiples of 4")
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4
        e = lambda n, h, w, c: torch.empty((n, h, w, c), dtype=torch.bfloat16, device=self.dev)  # noqa: E731
        b = {"x": e(N, H, W, 16), "a1a": e(N, H, W, 32), "cat1": e(N, H, W, 96), "p1": e(N, h2, w2, 32),
             "a2a": e(N, h2, w2, 64), "cat2": e(N, h2, w2, 192), "p2": e(N, h4, w4, 64), "a3a": e(N, h4, w4, 128),
             "a3b": e(N, h4, w4, 128), "a4a": e(N, h2, w2, 64), "a4b": e(N, h2, w2, 64), "a5a": e(N, H, W, 32),
             "a5b": e(N, H, W, 32), "out": e(N, H, W, 16),
             "out32": torch.empty((N, H, W, 16), dtype=torch.float32, device=self.dev),
             "base": torch.empty((N, H, W, 3), dtype=torch.float32, device=self.dev)}
        if train:
            for k in ("out", "a5b", "a5a", "cat1", "a4b", "a4a", "cat2", "a3b", "a3a", "p2", "a2a", "p1", "a1a"):
                b["g_" + k] = torch.zeros_like(b[k])
        self._bufs[key] = b
        return b

    # -- layer calls -----------------------------------------------------------------
    def _desc(self, N, H, W, cin, cout, xs, xo, ys, yo):
        return nat.ConvDesc(N, H, W, cin, cout, xs, xo, ys, yo)

    def _stream(self):
        # torch's default stream has handle 0; the library would read NULL as
        # its own (non-blocking) stream, so name the legacy default stream (1)
        h = _torch().cuda.current_stream(self.dev).cuda_stream
        return ctypes.c_void_p(h or 1)

    def _conv(self, name, N, H, W, x, xs, xo, y, ys, yo, y32=None):
        _, cin, cout, relu = next(L for L in LAYERS if L[0] == name)
        d = self._desc(N, H, W, cin, cout, xs, xo, ys, yo)
        self.ctx.check(nat.lib().rx_conv_bf16_fwd(self.ctx.h, ctypes.byref(d), _ptr(x), _ptr(self.w16[name]),
                                                  _ptr(self.b32[name]), _ptr(y), _ptr(y32), relu, self._stream()))

    def _conv_bwd(self, name, N, H, W, x, xs, xo, dy, ys, yo, dx=None):
        _, cin, cout, _ = next(L for L in LAYERS if L[0] == name)
        d = self._desc(N, H, W, cin, cout, xs, xo, ys, yo)
        L = nat.lib()
        self.ctx.check(L.rx_conv_bf16_bwd_weight(self.ctx.h, ctypes.byref(d), _ptr(dy), _ptr(x), _ptr(self.dw[name]),
                                                 _ptr(self.db[name]), self._stream()))
        if dx is not None:
            self.ctx.check(L.rx_conv_bf16_bwd_data(self.ctx.h, ctypes.byref(d), _ptr(dy), _ptr(self.w16[name]),
                                                   _ptr(self.rot), _ptr(dx), self._stream()))

    def _layer(self, kind, N, H, W, C, a, a_stride, a_off, b, b_stride, b_off, flag=0):
        op = nat.DnOp(kind, N, H, W, C, ctypes.c_void_p(a.data_ptr()), a_stride, a_off,
                      ctypes.c_void_p(b.data_ptr()), b_stride, b_off, flag)
        self.ctx.check(nat.lib().rx_dn_layer(self.ctx.h, ctypes.byref(op), self._stream()))

    # -- network -------------------------------------------------------------------
    def features(self, radiance, albedo, normal, depth, N, H, W, train=False):
        """Write the input layer from float32 device tensors (N, H, W, 3) /
        (N, H, W)."""
        b = self.buffers(N, H, W, train)
        P = N * H * W
        self.ctx.check(nat.lib().rx_dn_features(self.ctx.h, P, _ptr(radiance), _ptr(albedo), _ptr(normal),
                                                _ptr(depth), _ptr(b["x"]), _ptr(b["base"]), self._stream()))
        return b

    def forward(self, N, H, W, train=False):
        b = self.buffers(N, H, W, train)
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4
        c = self._conv
        c("e1a", N, H, W, b["x"], 16, 0, b["a1a"], 32, 0)
        c("e1b", N, H, W, b["a1a"], 32, 0, b["cat1"], 96, 64)           # skip 1 -> cat1[64:96]
        self._layer(nat.RX_DN_POOL, N, H, W, 32, b["cat1"], 96, 64, b["p1"], 32, 0)
        c("e2a", N, h2, w2, b["p1"], 32, 0, b["a2a"], 64, 0)
        c("e2b", N, h2, w2, b["a2a"], 64, 0, b["cat2"], 192, 128)      # skip 2 -> cat2[128:192]
        self._layer(nat.RX_DN_POOL, N, h2, w2, 64, b["cat2"], 192, 128, b["p2"], 64, 0)
        c("e3a", N, h4, w4, b["p2"], 64, 0, b["a3a"], 128, 0)
        c("e3b", N, h4, w4, b["a3a"], 128, 0, b["a3b"], 128, 0)
        self._layer(nat.RX_DN_UP, N, h4, w4, 128, b["a3b"], 128, 0, b["cat2"], 192, 0)
        c("d2a", N, h2, w2, b["cat2"], 192, 0, b["a4a"], 64, 0)
        c("d2b", N, h2, w2, b["a4a"], 64, 0, b["a4b"], 64, 0)
        self._layer(nat.RX_DN_UP, N, h2, w2, 64, b["a4b"], 64, 0, b["cat1"], 96, 0)
        c("d1a", N, H, W, b["cat1"], 96, 0, b["a5a"], 32, 0)
        c("d1b", N, H, W, b["a5a"], 32, 0, b["a5b"], 32, 0)
        c("head", N, H, W, b["a5b"], 32, 0, b["out"], 16, 0, y32=b["out32"])
        return b

    def backward(self, N, H, W):
        """Weight gradients (accumulated into dw / db) for the output gradient
        in g_out."""
        b = self.buffers(N, H, W, True)
        h2, w2, h4, w4 = H // 2, W // 2, H // 4, W // 4
        mask = lambda n, h, w, C, y, ys, yo, g, gs, go: self._layer(  # noqa: E731
            nat.RX_DN_RELU_MASK, n, h, w, C, y, ys, yo, g, gs, go)
        self._conv_bwd("head", N, H, W, b["a5b"], 32, 0, b["g_out"], 16, 0, b["g_a5b"])
        mask(N, H, W, 32, b["a5b"], 32, 0, b["g_a5b"], 32, 0)
        self._conv_bwd("d1b", N, H, W, b["a5a"], 32, 0, b["g_a5b"], 32, 0, b["g_a5a"])
        mask(N, H, W, 32, b["a5a"], 32, 0, b["g_a5a"], 32, 0)
        self._conv_bwd("d1a", N, H, W, b["cat1"], 96, 0, b["g_a5a"], 32, 0, b["g_cat1"])
        self._layer(nat.RX_DN_UP_BWD, N, h2, w2, 64, b["g_cat1"], 96, 0, b["g_a4b"], 64, 0)
        mask(N, h2, w2, 64, b["a4b"], 64, 0, b["g_a4b"], 64, 0)
        self._conv_bwd("d2b", N, h2, w2, b["a4a"], 64, 0, b["g_a4b"], 64, 0, b["g_a4a"])
        mask(N, h2, w2, 64, b["a4a"], 64, 0, b["g_a4a"], 64, 0)
        self._conv_bwd("d2a", N, h2, w2, b["cat2"], 192, 0, b["g_a4a"], 64, 0, b["g_cat2"])
        self._layer(nat.RX_DN_UP_BWD, N, h4, w4, 128, b["g_cat2"], 192, 0, b["g_a3b"], 128, 0)
        mask(N, h4, w4, 128, b["a3b"], 128, 0, b["g_a3b"], 128, 0)
        self._conv_bwd("e3b", N, h4, w4, b["a3a"], 128, 0, b["g_a3b"], 128, 0, b["g_a3a"])
        mask(N, h4, w4, 128, b["a3a"], 128, 0, b["g_a3a"], 128, 0)
        self._conv_bwd("e3a", N, h4, w4, b["p2"], 64, 0, b["g_a3a"], 128, 0, b["g_p2"])
        # skip 2 gradient: concat part + pooled path
        self._layer(nat.RX_DN_POOL_BWD, N, h2, w2, 64, b["g_p2"], 64, 0, b["g_cat2"], 192, 128, flag=1)
        mask(N, h2, w2, 64, b["cat2"], 192, 128, b["g_cat2"], 192, 128)
        self._conv_bwd("e2b", N, h2, w2, b["a2a"], 64, 0, b["g_cat2"], 192, 128, b["g_a2a"])
        mask(N, h2, w2, 64, b["a2a"], 64, 0, b["g_a2a"], 64, 0)
        self._conv_bwd("e2a", N, h2, w2, b["p1"], 32, 0, b["g_a2a"], 64, 0, b["g_p1"])
        self._layer(nat.RX_DN_POOL_BWD, N, H, W, 32, b["g_p1"], 32, 0, b["g_cat1"], 96, 64, flag=1)
        mask(N, H, W, 32, b["cat1"], 96, 64, b["g_cat1"], 96, 64)
        self._conv_bwd("e1b", N, H, W, b["a1a"], 32, 0, b["g_cat1"], 96, 64, b["g_a1a"])
        mask(N, H, W, 32, b["a1a"], 32, 0, b["g_a1a"], 32, 0)
        self._conv_bwd("e1a", N, H, W, b["x"], 16, 0, b["g_a1a"], 32, 0, None)

    def loss(self, N, H, W, target):
        """L1 loss (log1p space) of the current output against target
        (float32 device tensor (N, H, W, 3) of log1p radiance); writes g_out."""
        b = self.buffers(N, H, W, True)
        P = N * H * W
        self.loss_acc.zero_()
        self.ctx.check(nat.lib().rx_dn_l1_loss(self.ctx.h, P, _ptr(b["out32"]), 16, _ptr(b["base"]), _ptr(target),
                                               ctypes.c_float(1.0 / (3 * P)), _ptr(b["g_out"]), 16,
                                               _ptr(self.loss_acc), self._stream()))
        return self.loss_acc

    def adam(self, lr=2e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        L = nat.lib()
        for name, _, _, _ in LAYERS:
            n = self.w32[name].numel()
            self.ctx.check(L.rx_dn_adam(self.ctx.h, n, _ptr(self.w32[name]), _ptr(self.dw[name]), _ptr(self.mw[name]),
                                        _ptr(self.vw[name]), _ptr(self.w16[name]), lr, b1, b2, eps, self.step,
                                        self._stream()))
            self.ctx.check(L.rx_dn_adam(self.ctx.h, self.b32[name].numel(), _ptr(self.b32[name]), _ptr(self.db[name]),
                                        _ptr(self.mb[name]), _ptr(self.vb[name]), None, lr, b1, b2, eps, self.step,
                                        self._stream()))

    def train_step(self, radiance, albedo, normal, depth, target, lr=2e-3):
        N, H, W = radiance.shape[:3]
        self.features(radiance, albedo, normal, depth, N, H, W, train=True)
        self.forward(N, H, W, train=True)
        loss = self.loss(N, H, W, target)
        self.backward(N, H, W)
        self.adam(lr)
        return loss

    def denoise(self, radiance, albedo, normal, depth):
        """Denoised linear radiance (N, H, W, 3) float32 device tensor from
        float32 device tensors; H and W multiples of 4."""
        torch = _torch()
        N, H, W = radiance.shape[:3]
        b = self.features(radiance, albedo, normal, depth, N, H, W)
        self.forward(N, H, W)
        out = torch.empty((N, H, W, 3), dtype=torch.float32, device=self.dev)
        self.ctx.check(nat.lib().rx_dn_output(self.ctx.h, N * H * W, _ptr(b["out32"]), 16, _ptr(b["base"]), _ptr(out),
                                              self._stream()))
        return out


# -- training data from the renderer -----------------------------------------------
def render_views(scene_world, device_scene, views, size, spp, max_depth=12, seed=0, ref=False):
    """Render `views` (list of (cam_pos, look_at)) at size x size; returns a
    dict of float32 arrays (V, size, size, 3|1): radiance, albedo, normal,
    depth (the float64 mean for ref=True)."""
    from rendering.taichi.trace import make_params
    cam = scene_world.active_camera
    out = {k: [] for k in ("radiance", "albedo", "normal", "depth")}
    acc = nat.Accumulator(size, size)
    for i, (at_pos, at) in enumerate(views):
        pos, fwd, right, up = _look_at(at_pos, at)
        p = make_params(size, size, math.tan(math.radians(cam.fov) / 2), 1.0, max_depth, int(scene_world._use_sky), 0,
                        1, 10.0, list(scene_world._background_color), pos, fwd, right, up, seed=seed + i)
        acc.reset()
        if ref:
            acc.set_f64(True)
        acc.render(device_scene.native, p, spp)
        out["radiance"].append(acc.read_f64().astype(np.float32) if ref else acc.read(nat.RX_ACC_RADIANCE))
        out["albedo"].append(acc.read(nat.RX_ACC_ALBEDO))
        out["normal"].append(acc.read(nat.RX_ACC_NORMAL))
        out["depth"].append(acc.read(nat.RX_ACC_DEPTH)[..., None])
        if ref:
            acc.set_f64(False)
    acc.close()
    return {k: np.stack(v) for k, v in out.items()}


WEIGHTS = __file__.rsplit("/", 1)[0] + "/denoiser_weights.npz"


def save_weights(net, path):
    """Weights as bf16 bit patterns (what inference reads), biases float32."""
    out = {}
    for name, _, _, _ in LAYERS:
        w = net.w32[name].cpu().numpy().astype(np.float32)
        out[f"{name}.w16"] = (w.view(np.uint32) + 0x7FFF + ((w.view(np.uint32) >> 16) & 1) >> 16).astype(np.uint16)
        out[f"{name}.b"] = net.b32[name].cpu().numpy()
    np.savez_compressed(path, **out)


def load_weights(path=WEIGHTS):
    d = np.load(path)
    out = {}
    for name, _, _, _ in LAYERS:
        out[f"{name}.w"] = (d[f"{name}.w16"].astype(np.uint32) << 16).view(np.float32)
        out[f"{name}.b"] = d[f"{name}.b"]
    return out


def make_training_set(scene_seeds=(3001, 3002, 3003, 3004), views_per_scene=48, size=256, spp_in=4, spp_ref=256,
                      seed=5):
    """Noisy / reference pairs rendered from orbiting cameras over scenes of
    the large-mesh generator (other seeds than the evaluation scene).
    Returns float32 numpy arrays: radiance, albedo, normal, depth (V, S, S,
    3|1) of the noisy renders and target (V, S, S, 3) = log1p(reference)."""
    import workloads
    from rendering.taichi.extractor import build_device_scene
    parts = {k: [] for k in ("radiance", "albedo", "normal", "depth", "target")}
    for k, s in enumerate(scene_seeds):
        world = workloads.displaced_icosphere_scene(size, size, seed=s)
        ds = build_device_scene(world)
        ds.use_lights(False)
        views = orbit_views(views_per_scene, seed + k)
        noisy = render_views(world, ds, views, size, spp_in, seed=1000 * k + 17)
        ref = render_views(world, ds, views, size, spp_ref, seed=1000 * k + 500000, ref=True)
        for key in ("radiance", "albedo", "normal", "depth"):
            parts[key].append(noisy[key])
        parts["target"].append(np.log1p(np.maximum(ref["radiance"], 0.0)).astype(np.float32))
    return {k: np.concatenate(v) for k, v in parts.items()}


def train(net, data, steps=3000, batch=16, crop=128, lr=2e-3, seed=0, log_every=250):
    """Adam on random crops (with flips) of the training set held on the
    device; the learning rate decays by a cosine to 5 % of `lr`.  Returns the
    loss history (mean L1 in log1p space per logged step)."""
    torch = _torch()
    dev = net.dev
    T = {k: torch.from_numpy(v).to(dev) for k, v in data.items()}
    V, S = T["radiance"].shape[:2]
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    acc = 0.0
    for it in range(steps):
        idx = torch.randint(0, V, (batch,), generator=g)
        oy = torch.randint(0, S - crop + 1, (1,), generator=g).item() // 4 * 4
        ox = torch.randint(0, S - crop + 1, (1,), generator=g).item() // 4 * 4
        flip = torch.randint(0, 4, (1,), generator=g).item()

        def pick(t):
            c = t[idx.to(dev), oy:oy + crop, ox:ox + crop]
            if flip & 1:
                c = torch.flip(c, (2,))
            if flip & 2:
                c = torch.flip(c, (1,))
            return c.contiguous()

        # normals are world-space guides: mirrored crops keep them as rendered
        rad, alb, nrm, dep, tgt = (pick(T[k]) for k in ("radiance", "albedo", "normal", "depth", "target"))
        cur = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * it / max(steps, 1))))
        loss = net.train_step(rad, alb, nrm, dep, tgt, lr=cur)
        acc += float(loss) / (3 * batch * crop * crop)
        if (it + 1) % log_every == 0:
            hist.append(acc / log_every)
            acc = 0.0
    return hist


def _look_at(pos, at):
    pos = np.asarray(pos, np.float64)
    fwd = np.asarray(at, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    return list(pos), list(fwd), list(right), list(np.cross(right, fwd))


def evaluate(net, world, width=1920, height=1080, spp=4, ref_spp=4096, max_depth=12, seed=77, view=None):
    """relMSE of the noisy render, the 5-pass a-trous filter and the learned
    denoiser against a float64 `ref_spp` render of the same view (the
    world's camera, or `view` = (position, look-at point)); plus the learned
    denoiser's inference time (CUDA events, mean of 10 after 3)."""
    torch = _torch()
    from rendering.quality import reference_render, rel_mse
    from rendering.taichi.extractor import build_device_scene
    from rendering.taichi.trace import make_params
    cam = world.active_camera
    ds = build_device_scene(world)
    ds.use_lights(False)
    if view is None:
        pos, fwd, right, up = list(cam.position), list(cam.forward), list(cam.right), list(cam.up)
    else:
        pos, fwd, right, up = _look_at(*view)
    p = make_params(width, height, math.tan(math.radians(cam.fov) / 2), cam.aspect_ratio, max_depth,
                    int(world._use_sky), 0, 1, 10.0, list(world._background_color), pos, fwd, right, up, seed=seed)
    ref = reference_render(ds.native, p, ref_spp)
    acc = nat.Accumulator(width, height)
    acc.render(ds.native, p, spp)
    noisy = acc.read(nat.RX_ACC_RADIANCE)
    dp = nat.DenoiseParams(1, 5, 0.08, 0.35, 0.20, 1.0, 1.0, 1, 1, 1, 0)
    atrous = acc.denoise(dp)
    dev = net.dev
    planes = [torch.from_numpy(acc.read(w)).to(dev)[None] for w in
              (nat.RX_ACC_RADIANCE, nat.RX_ACC_ALBEDO, nat.RX_ACC_NORMAL)]
    dep = torch.from_numpy(acc.read(nat.RX_ACC_DEPTH)).to(dev)[None, ..., None].contiguous()
    out = net.denoise(*planes, dep)
    for _ in range(3):
        net.denoise(*planes, dep)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        net.denoise(*planes, dep)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / 10
    learned = out[0].cpu().numpy()
    flops = 2.0 * macs_per_pixel() * width * height
    return {"relmse_noisy": rel_mse(noisy, ref), "relmse_atrous": rel_mse(atrous, ref),
            "relmse_learned": rel_mse(learned, ref), "spp": spp, "ref_spp": ref_spp, "infer_ms": ms,
            "infer_tflops": flops / (ms / 1e3) / 1e12, "flops_per_frame": flops}


HELD_OUT_SEEDS = tuple(range(4001, 4009))  # scene seeds never rendered for training


def evaluate_held_out(net, seeds=HELD_OUT_SEEDS, spp=4, ref_spp=4096):
    """`evaluate` on one orbit view of each held-out scene of the large-mesh
    generator at 1920x1080: per-view relMSE of the noisy render, the a-trous
    filter and the learned denoiser, and their means."""
    import workloads
    rows = []
    for k, s in enumerate(seeds):
        view = orbit_views(1, 9000 + s)[0]
        r = evaluate(net, workloads.displaced_icosphere_scene(seed=s), spp=spp, ref_spp=ref_spp, seed=500 + k,
                     view=view)
        rows.append({"seed": s, **{m: r[m] for m in ("relmse_noisy", "relmse_atrous", "relmse_learned")}})
    mean = {m: float(np.mean([r[m] for r in rows])) for m in ("relmse_noisy", "relmse_atrous", "relmse_learned")}
    return {"views": rows, "mean": mean, "spp": spp, "ref_spp": ref_spp}


def main():
    """Train on renderer-generated pairs and write the weights file."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--scenes", type=int, default=16, help="training scenes (seeds 3001, 3002, ...)")
    ap.add_argument("--views", type=int, default=128, help="orbit views per training scene")
    ap.add_argument("--spp-ref", type=int, default=1024, help="spp of the training targets")
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--eval", action="store_true")
    ap.add_argument("--infer", default=None, metavar="WxH",
                    help="only run `--repeat` inferences of the committed weights on seeded random WxH inputs "
                         "(the kernel-profiling case) and exit")
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    if args.infer:
        torch = _torch()
        w, h = (int(v) for v in args.infer.lower().split("x"))
        net = Denoiser(weights=load_weights())
        g = torch.Generator(device=net.dev).manual_seed(1)
        planes = [torch.rand((1, h, w, 3), generator=g, device=net.dev) for _ in range(3)]
        dep = torch.rand((1, h, w, 1), generator=g, device=net.dev)
        for _ in range(args.repeat):
            net.denoise(*planes, dep)
        torch.cuda.synchronize()
        net.ctx.check(nat.lib().rx_ctx_sync(net.ctx.h))
        print(json.dumps({"infer": [w, h], "repeat": args.repeat}))
        return
    t0 = time.time()
    data = make_training_set(scene_seeds=tuple(range(3001, 3001 + args.scenes)), views_per_scene=args.views,
                             spp_ref=args.spp_ref)
    t_data = time.time() - t0
    net = Denoiser(seed=0)
    t0 = time.time()
    hist = train(net, data, steps=args.steps)
    t_train = time.time() - t0
    save_weights(net, args.out)
    res = {"pairs": int(data["radiance"].shape[0]), "spp_ref": args.spp_ref, "data_s": t_data, "train_s": t_train,
           "loss": hist}
    if args.eval:
        import workloads
        net2 = Denoiser(weights=load_weights(args.out))
        res["eval"] = evaluate(net2, workloads.displaced_icosphere_scene())
        res["held_out"] = evaluate_held_out(net2)
    print(json.dumps(res))


def orbit_views(n, seed, radius=(2.4, 3.6)):
    """Seeded camera positions around the scene's centre, looking at it."""
    rng = np.random.default_rng(seed)
    views = []
    for _ in range(n):
        az = rng.uniform(0, 2 * np.pi)
        el = rng.uniform(-0.2, 0.7)
        r = rng.uniform(*radius)
        pos = [r * math.cos(el) * math.sin(az), r * math.sin(el) + 0.3, r * math.cos(el) * math.cos(az)]
        at = rng.normal(0.0, 0.25, 3).tolist()
        views.append((pos, at))
    return views


if __name__ == "__main__":
    main()
