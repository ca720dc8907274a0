from core import Color


class World:
    """Objects, cameras, sky / background (the active camera is the first added)."""

    def __init__(self, objects=None, lights=None, cameras=None, background_color=None, use_sky=True):
        self._objects = objects if objects is not None else []
        self._lights = lights if lights is not None else []
        self._cameras = cameras if cameras is not None else []
        self._background_color = background_color if background_color is not None else Color(0, 0, 0)
        self._use_sky = use_sky
        self._active_camera = self._cameras[0] if self._cameras else None

    def add_object(self, obj):
        self._objects.append(obj)

    def add_camera(self, camera):
        self._cameras.append(camera)
        if not self._active_camera:
            self._active_camera = camera

    def remove_object(self, obj):
        self._objects.remove(obj)

    objects = property(lambda s: s._objects)
    cameras = property(lambda s: s._cameras)
    lights = property(lambda s: s._lights)

    @property
    def active_camera(self):
        return self._active_camera

    @active_camera.setter
    def active_camera(self, cam):
        if cam not in self._cameras:
            raise ValueError("Camera must be added to the world before it can be set as active.")
        self._active_camera = cam

    @property
    def use_sky(self):
        return self._use_sky

    @use_sky.setter
    def use_sky(self, v):
        self._use_sky = v

    @property
    def background_color(self):
        return self._background_color

    @background_color.setter
    def background_color(self, c):
        self._background_color = c
