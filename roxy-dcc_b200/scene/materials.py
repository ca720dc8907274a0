"""Surface materials.  Type ids and parameters are the GPU contract of the
reference (scene/materials.py taichi_type_id / taichi_params):
0 diffuse, 1 metal (roughness), 2 dielectric (ior), 3 emissive (intensity),
4 glossy (roughness)."""
from core import Color


class Material:
    def __init__(self, albedo=None, albedo_texture=None):
        self._albedo = albedo or Color(1, 1, 1)
        self._albedo_texture = albedo_texture

    def taichi_type_id(self):
        return 0

    def taichi_params(self):
        return []


class Diffuse(Material):
    def __init__(self, albedo, albedo_texture=None):
        super().__init__(albedo, albedo_texture)

    def __repr__(self):
        return f"Diffuse(albedo={self._albedo})"


class Metal(Material):
    def __init__(self, albedo, roughness=0.0, albedo_texture=None):
        super().__init__(albedo, albedo_texture)
        self._roughness = min(max(roughness, 0.0), 1.0)

    def taichi_type_id(self):
        return 1

    def taichi_params(self):
        return [self._roughness]


class Dielectric(Material):
    def __init__(self, albedo, ior=1.5, albedo_texture=None):
        super().__init__(albedo, albedo_texture)
        self._ior = ior

    def taichi_type_id(self):
        return 2

    def taichi_params(self):
        return [self._ior]


class Emissive(Material):
    def __init__(self, color, intensity=1.0, albedo_texture=None):
        super().__init__(color, albedo_texture)
        self._intensity = intensity

    def emitted(self):
        return self._albedo * self._intensity

    def taichi_type_id(self):
        return 3

    def taichi_params(self):
        return [self._intensity]


class Glossy(Material):
    def __init__(self, albedo, roughness=0.5, albedo_texture=None):
        super().__init__(albedo, albedo_texture)
        self._roughness = min(max(roughness, 0.0), 1.0)

    def taichi_type_id(self):
        return 4

    def taichi_params(self):
        return [self._roughness]
