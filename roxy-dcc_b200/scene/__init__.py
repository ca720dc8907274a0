"""Scene object model consumed by the renderer (same API as roxy-dcc's scene package)."""
from scene.camera import Camera
from scene.materials import Dielectric, Diffuse, Emissive, Glossy, Material, Metal
from scene.mesh import IndexedMesh, Mesh, Triangle
from scene.primitives import Cube, Plane, Primitive, Sphere
from scene.scene_object import SceneObject
from scene.shape import Shape
from scene.textures import ImageTexture
from scene.world import World

__all__ = ["Camera", "Dielectric", "Diffuse", "Emissive", "Glossy", "Material", "Metal", "IndexedMesh", "Mesh",
           "Triangle", "Cube", "Plane", "Primitive", "Sphere", "SceneObject", "Shape", "ImageTexture", "World"]
