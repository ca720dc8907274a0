class ImageTexture:
    """Albedo texture handle (path + flip flag).  Textured albedo is not yet
    sampled on the GPU path; materials carrying one render with their base
    albedo."""

    def __init__(self, path=None, flip_v=False):
        self.path = path
        self.flip_v = flip_v
