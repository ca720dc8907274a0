"""GPU path (names kept from the reference's Taichi package)."""
from rendering.taichi.bvh_builder import GPUBVHBuilder, TriangleBatch
from rendering.taichi.extractor import extract_scene
from rendering.taichi.fields import MAX_H, MAX_W
from rendering.taichi.trace import render_kernel

__all__ = ["GPUBVHBuilder", "TriangleBatch", "extract_scene", "render_kernel", "MAX_W", "MAX_H"]
