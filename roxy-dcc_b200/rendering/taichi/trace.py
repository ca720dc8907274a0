"""render_kernel: one progressive frame with the reference's argument list
(rendering/taichi/trace.py:239-254), run as the wavefront CUDA render on the
scene bound by extract_scene."""
import roxy_native as nat
from rendering.taichi import fields


def make_params(W, H, fov_tan, aspect, max_depth, use_sky, direct_light_mode, direct_light_max_depth, sample_clamp,
                bg_color, cam_pos, cam_fwd, cam_right, cam_up, reference_compat=False, seed=0, wave_paths=0,
                mis=False):
    p = nat.RenderParams()
    p.width, p.height = int(W), int(H)
    p.fov_tan, p.aspect = float(fov_tan), float(aspect)
    for name, v in (("cam_pos", cam_pos), ("cam_fwd", cam_fwd), ("cam_right", cam_right), ("cam_up", cam_up),
                    ("bg", bg_color)):
        arr = getattr(p, name)
        vals = list(v)
        for k in range(3):
            arr[k] = float(vals[k])
    p.max_depth, p.use_sky = int(max_depth), int(bool(use_sky))
    p.direct_light_mode, p.direct_light_max_depth = int(direct_light_mode), int(direct_light_max_depth)
    p.sample_clamp = float(sample_clamp) if sample_clamp is not None else 0.0
    p.reference_compat, p.seed, p.wave_paths = int(bool(reference_compat)), int(seed) & 0xFFFFFFFF, int(wave_paths)
    p.mis = int(bool(mis))
    return p


def render_kernel(W, H, fov_tan, aspect, max_depth, use_sky, direct_light_mode, direct_light_max_depth,
                  sample_clamp, count_rays, bg_color, cam_pos, cam_fwd, cam_right, cam_up):
    ds = fields.current_scene()
    if ds is None:
        raise RuntimeError("render_kernel: call extract_scene(world) first")
    ds.use_lights(False)
    acc = fields.accumulator(W, H)
    p = make_params(W, H, fov_tan, aspect, max_depth, use_sky, direct_light_mode, direct_light_max_depth,
                    sample_clamp, bg_color, cam_pos, cam_fwd, cam_right, cam_up)
    acc.render(ds.native, p, 1)
