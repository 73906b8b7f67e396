"""Minimal stand-in for fv3gfs.util (fixture generation only).

Provides the dimension names, the sub-tile sizer, a light Quantity and the
type names that the reference's hot-path modules import.  Halo exchange is
not here: the fixture generator supplies its own communicator object.
"""
import dataclasses
from typing import Any, Sequence, Tuple

import numpy as np

from . import constants, halo_data_transformer  # noqa: F401
from .constants import *  # noqa: F401,F403
from .constants import X_DIMS, Y_DIMS, Z_DIMS, X_INTERFACE_DIM, Y_INTERFACE_DIM, Z_INTERFACE_DIM


class SubtileGridSizer:
    def __init__(self, nx, ny, nz, n_halo, extra_dim_lengths=None):
        self.nx, self.ny, self.nz, self.n_halo = nx, ny, nz, n_halo
        self.extra_dim_lengths = extra_dim_lengths or {}

    def get_extent(self, dims):
        out = []
        for d in dims:
            if d in X_DIMS:
                out.append(self.nx + (1 if d == X_INTERFACE_DIM else 0))
            elif d in Y_DIMS:
                out.append(self.ny + (1 if d == Y_INTERFACE_DIM else 0))
            elif d in Z_DIMS:
                out.append(self.nz + (1 if d == Z_INTERFACE_DIM else 0))
            else:
                out.append(self.extra_dim_lengths[d])
        return tuple(out)

    def get_origin(self, dims):
        return tuple(self.n_halo if (d in X_DIMS or d in Y_DIMS) else 0 for d in dims)


GridSizer = SubtileGridSizer


@dataclasses.dataclass
class QuantityMetadata:
    origin: Tuple[int, ...]
    extent: Tuple[int, ...]
    dims: Tuple[str, ...]
    units: str
    dtype: Any


class Quantity:
    def __init__(self, data, dims, units="unknown", origin=None, extent=None, gt4py_backend=None):
        self.data = data
        self.storage = data
        self.np = np
        if origin is None:
            origin = (0,) * len(dims)
        if extent is None:
            extent = tuple(s - o for s, o in zip(np.shape(data), origin))
        self.metadata = QuantityMetadata(tuple(origin), tuple(extent), tuple(dims), units, np.float64)
        self.dims = tuple(dims)
        self.origin = tuple(origin)
        self.extent = tuple(extent)
        self.units = units

    @property
    def view(self):
        return self


class TilePartitioner:
    def __init__(self, layout):
        self.layout = layout

    def subtile_index(self, rank):
        return (0, 0)


class CubedSphereCommunicator:  # type name only
    pass


class Timer:
    def clock(self, name):
        import contextlib

        return contextlib.nullcontext()


NullTimer = Timer


class QuantityFactory:
    @classmethod
    def from_backend(cls, sizer, backend=None):
        return cls()
