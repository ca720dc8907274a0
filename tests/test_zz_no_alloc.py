"""rx_denoise_noalloc: the denoise entry point for callers that cannot
allocate device memory at call time (a host application that owns the whole
device budget through its own allocator, or a frame loop that must not pay
an allocation's implicit synchronisation).  Its output must equal the
allocating entry point's (rx_denoise) on the same inputs, call after call,
even though every call reuses the same fixed scratch array.

The test allocates its own buffers (with torch); the entry point under test
allocates nothing.  This file is collected last so a failure here cannot
stop the rest of a -x run early.
"""
import ctypes

import numpy as np
import pytest

import roxy_native as nat

pytestmark = pytest.mark.gpu


def _inputs(seed, H, W):
    rng = np.random.default_rng(seed)
    color = (rng.random((H, W, 3)) * 2.0).astype(np.float32)
    normal = rng.normal(size=(H, W, 3)).astype(np.float32)
    normal /= np.linalg.norm(normal, axis=2, keepdims=True)
    normal[: H // 3] = [0.0, 1.0, 0.0]
    albedo = rng.random((H, W, 3)).astype(np.float32)
    depth = (rng.random((H, W)) * 3.0 + 1.0).astype(np.float32)
    return color, normal, albedo, depth


def _pack4(torch, rgb, w=None):
    H, W = rgb.shape[:2]
    a = np.zeros((H, W, 4), np.float32)
    a[..., :3] = rgb
    if w is not None:
        a[..., 3] = w
    return torch.from_numpy(a).cuda()


def test_noalloc_denoise_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    L = nat.lib()
    nat.context()  # the allocating reference path below needs a context
    stream = torch.cuda.current_stream()
    for call, (seed, H, W, passes, radius) in enumerate(((1, 96, 130, 3, 1), (2, 77, 61, 5, 2))):
        color, normal, albedo, depth = _inputs(seed, H, W)
        ref = nat.denoise(color, normal=normal, albedo=albedo, depth=depth, radius=radius, sigma_color=0.1,
                          amount=0.8, passes=passes)
        c4 = _pack4(torch, color)
        n4 = _pack4(torch, normal, depth)
        a4 = _pack4(torch, albedo)
        out = torch.full((H, W, 4), float("nan"), device="cuda")
        p = nat.DenoiseParams(radius, passes, 0.1, 0.35, 0.20, 1.0, 0.8, 1, 1, 1, 0)
        rc = L.rx_denoise_noalloc(H, W, c4.data_ptr(), n4.data_ptr(), a4.data_ptr(), ctypes.byref(p),
                                  out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == nat.RX_OK, L.rx_last_error(None)
        torch.cuda.synchronize()
        got = out[..., :3].cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=2e-6, atol=2e-6, err_msg=f"call {call}")


def test_noalloc_denoise_rejects_sizes_beyond_its_scratch():
    L = nat.lib()
    p = nat.DenoiseParams(1, 2, 0.1, 0.35, 0.20, 1.0, 0.8, 0, 0, 0, 0)
    # no buffer is touched: the size check comes before any launch
    rc = L.rx_denoise_noalloc(1025, 1024, None, None, None, ctypes.byref(p), None, None)
    assert rc == nat.RX_ERR_CAPACITY
    assert b"scratch limit" in L.rx_last_error(None)


def _noalloc(torch, L, H, W, c4, n4, a4, p, out):
    rc = L.rx_denoise_noalloc(H, W, c4.data_ptr(), n4.data_ptr() if n4 is not None else None,
                              a4.data_ptr() if a4 is not None else None, ctypes.byref(p), out.data_ptr(),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == nat.RX_OK, L.rx_last_error(None)
    torch.cuda.synchronize()
    return out[..., :3].cpu().numpy()


def test_noalloc_copy_path_and_guides_off():
    """radius 0 (the display copy) and a filter with every guide off and NULL
    guide pointers, each against the allocating entry point."""
    torch = pytest.importorskip("torch")
    L = nat.lib()
    nat.context()
    H, W = 40, 57
    color, normal, albedo, depth = _inputs(5, H, W)
    c4 = _pack4(torch, color)
    out = torch.full((H, W, 4), float("nan"), device="cuda")
    p = nat.DenoiseParams(0, 1, 0.1, 0.35, 0.20, 1.0, 0.8, 0, 0, 0, 1)
    got = _noalloc(torch, L, H, W, c4, None, None, p, out)
    np.testing.assert_array_equal(got, np.sqrt(np.clip(color, 0.0, 1.0)))
    for passes in (1, 4):
        ref = nat.denoise(color, radius=1, sigma_color=0.2, amount=0.9, passes=passes)
        p = nat.DenoiseParams(1, passes, 0.2, 0.35, 0.20, 1.0, 0.9, 0, 0, 0, 0)
        out.fill_(float("nan"))
        got = _noalloc(torch, L, H, W, c4, None, None, p, out)
        np.testing.assert_allclose(got, ref, rtol=2e-6, atol=2e-6, err_msg=f"{passes} passes, no guides")


def test_noalloc_rejects_an_output_that_overlaps_an_input():
    torch = pytest.importorskip("torch")
    L = nat.lib()
    H, W = 8, 8
    c4 = torch.zeros((H, W, 4), device="cuda")
    n4 = torch.zeros((H, W, 4), device="cuda")
    p = nat.DenoiseParams(1, 2, 0.1, 0.35, 0.20, 1.0, 0.8, 1, 0, 0, 0)
    for out in (c4, n4):
        rc = L.rx_denoise_noalloc(H, W, c4.data_ptr(), n4.data_ptr(), None, ctypes.byref(p), out.data_ptr(), None)
        assert rc == nat.RX_ERR_ARG
        assert b"overlap" in L.rx_last_error(None)
