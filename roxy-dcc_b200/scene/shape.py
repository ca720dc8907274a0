class Shape:
    """Geometry plus a group-name -> material mapping."""

    def __init__(self, geometry, material_groups=None, name=""):
        self._geometry = geometry
        self._material_groups = material_groups or {}
        self._default_material = None
        self._name = name

    geometry = property(lambda s: s._geometry)
    material_groups = property(lambda s: s._material_groups)
    name = property(lambda s: s._name)

    def set_default_material(self, material):
        self._default_material = material

    def material_for_group(self, group_name):
        return self._material_groups.get(group_name) or self._default_material

    @property
    def is_infinite(self):
        return getattr(self._geometry, "is_infinite", False)
