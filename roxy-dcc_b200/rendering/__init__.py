"""Rendering entry points (same module layout as roxy-dcc's rendering package)."""
from rendering.image import Image
from rendering.ray_tracer import RayTracer
from rendering.render_stats import RenderStats

__all__ = ["Image", "RayTracer", "RenderStats"]
