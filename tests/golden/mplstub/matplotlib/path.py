"""Stand-in for ``matplotlib.path``; polygon voxelisation is not used by any fixture."""


class Path:
    def __init__(self, *args, **kwargs):
        raise NotImplementedError("polygon masks need the real matplotlib")
