"""Wavefront MTL material libraries (scene/io/mtl_loader.py:1-97): the
parsed record and its mapping to the renderer's materials."""
from dataclasses import dataclass
from pathlib import Path

from core import Color
from scene.materials import Dielectric, Diffuse, Emissive, Glossy, Metal
from scene.textures import ImageTexture


@dataclass
class MTLMaterial:
    name: str
    ka: Color = None   # ambient
    kd: Color = None   # diffuse
    ks: Color = None   # specular
    ke: Color = None   # emissive
    tf: Color = None   # transmission filter
    ns: float = 10.0   # shininess
    ni: float = 1.0    # index of refraction
    d: float = 1.0     # opacity
    tr: float = 0.0    # transparency (1 - d)
    illum: int = 1     # illumination model
    map_kd: str = None  # diffuse texture path

    def to_material(self):
        """Material chosen as mtl_loader.py:24-38 does: emission first, then
        transparency (d < 0.99), illum 3-5 metals, a specular colour
        (glossy), else diffuse; roughness = max(0, 1 - Ns / 1000)."""
        texture = ImageTexture(self.map_kd) if self.map_kd else None
        if self.ke and (self.ke.r > 0 or self.ke.g > 0 or self.ke.b > 0):
            return Emissive(self.ke, intensity=1.0, albedo_texture=texture)
        if self.d < 0.99:
            return Dielectric(self.tf if self.tf else Color(1, 1, 1), ior=self.ni, albedo_texture=texture)
        if self.illum in (3, 4, 5):
            return Metal(self.kd or Color(1, 1, 1), roughness=max(0.0, 1.0 - self.ns / 1000.0),
                         albedo_texture=texture)
        if self.ks and (self.ks.r > 0 or self.ks.g > 0 or self.ks.b > 0):
            return Glossy(self.kd or Color(1, 1, 1), roughness=max(0.0, 1.0 - self.ns / 1000.0),
                          albedo_texture=texture)
        return Diffuse(self.kd or Color(0.8, 0.8, 0.8), albedo_texture=texture)


_COLORS = {"Ka": "ka", "Kd": "kd", "Ks": "ks", "Ke": "ke", "Tf": "tf"}


class MTLLoader:
    @staticmethod
    def load(path) -> dict:
        """{name: MTLMaterial} of a .mtl file (mtl_loader.py:41-97): full-line
        comments are skipped, text after '#' is dropped, keywords are
        case-sensitive, `map_Kd` keeps its last token joined to the file's
        directory, `Tr` sets d = 1 - Tr."""
        base_dir = Path(path).parent
        materials = []
        cur = None
        with open(path, "r") as f:
            for line in f:
                if line.startswith("#"):
                    continue
                parts = line.rsplit("#")[0].split()
                if not parts:
                    continue
                key = parts[0]
                if key == "newmtl":
                    if cur:
                        materials.append(cur)
                    cur = MTLMaterial(name=parts[1])
                if key == "Ns":
                    cur.ns = float(parts[1])
                if key == "Ni":
                    cur.ni = float(parts[1])
                if key == "d":
                    cur.d = float(parts[1])
                if key == "Tr":
                    cur.tr = float(parts[1])
                    cur.d = 1.0 - cur.tr
                if key == "illum":
                    cur.illum = int(parts[1])
                if key in ("map_kd", "map_Kd"):
                    cur.map_kd = str(base_dir / parts[-1])
                if key in _COLORS:
                    r, g, b = parts[1:]
                    setattr(cur, _COLORS[key], Color(float(r), float(g), float(b)))
        if cur:
            materials.append(cur)
        return {m.name: m for m in materials}
