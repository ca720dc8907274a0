"""The C-ABI library loads and exports every entry point include/roxy.h declares
(no device needed; nothing here launches a kernel)."""
import os
import re

import pytest

import roxy_native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "roxy.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|const char\*)\s+(rx_\w+)\s*\(", src, re.M)))


def test_header_declares_the_api():
    names = _declared()
    for n in ("rx_ctx_create", "rx_scene_set_triangles", "rx_bvh_build", "rx_trace_closest", "rx_render",
              "rx_accum_denoise", "rx_denoise"):
        assert n in names


@pytest.fixture(scope="module")
def L():
    if not os.path.exists(nat.LIB_PATH):
        nat.build()
    return nat.load_library()


def test_library_exports_every_declared_symbol(L):
    for name in _declared():
        assert hasattr(L, name), name


def test_binding_declares_every_symbol():
    assert set(_declared()) == set(nat._SIGS)


def test_binding_argument_counts_match_header():
    src = open(os.path.join(ROOT, "include", "roxy.h")).read()
    decls = re.findall(r"^\s*(?:int|void\*|const char\*)\s+(rx_\w+)\s*\(([^;]*?)\)\s*;", src, re.M | re.S)
    assert decls
    for name, params in decls:
        params = params.strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        assert len(nat._SIGS[name][0]) == n, f"{name}: header {n} args, binding {len(nat._SIGS[name][0])}"


def test_errors_without_device_are_reported_not_raised(L):
    import ctypes
    n = ctypes.c_int(-1)
    L.rx_device_count(ctypes.byref(n))
    assert n.value >= 0
    assert L.rx_version() >= 1
