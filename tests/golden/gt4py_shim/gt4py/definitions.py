import enum


class AccessKind(enum.IntFlag):
    NONE = 0
    READ = 1
    WRITE = 2
    READ_WRITE = 3


class FieldInfo:
    def __init__(self, access=None, boundary=None, axes=(), data_dims=(), dtype=None):
        self.access = access
        self.boundary = boundary
        self.axes = tuple(axes)
        self.data_dims = data_dims
        self.dtype = dtype
