"""The grid's metric terms generated on the GPU (``fv3b_generate_grid``).

``DeviceGrid`` plays the role of ``CubedSphereGrid`` (the numpy generator in
``grid.py``) for ``GridData``: the same fields, to rounding, computed point
by point on the device (the reference computes them in ``MetricTerms``,
fv3core/grid/generation.py:66, on the host).  Its 2-D fields are FP64
device tensors already in the stage kernels' layout ``[6, j, i]`` (i
fastest), so ``GridData`` takes them without a host round trip; the edge
weights are ``[6, n+1]`` and the corner ratios ``[6, 4, 3]``, as in
``CubedSphereGrid``.
"""
import ctypes

import torch

from . import _lib, constants
from .grid import LATTICES

# the order of fv3b_grid_fields.field (include/fv3core_b200.h)
GRID_FIELD_NAMES = [
    "dx", "dy", "dxa", "dya", "dxc", "dyc",
    "rdx", "rdy", "rdxa", "rdya", "rdxc", "rdyc",
    "area", "rarea", "area_c", "rarea_c",
    "sin_sg1", "sin_sg2", "sin_sg3", "sin_sg4", "sin_sg5",
    "cos_sg1", "cos_sg2", "cos_sg3", "cos_sg4", "cos_sg5",
    "cosa", "sina", "rsina",
    "cosa_u", "cosa_v", "cosa_s", "sina_u", "sina_v", "rsin_u", "rsin_v", "rsin2",
    "del6_u", "del6_v", "divg_u", "divg_v",
    "fC", "f0", "agrid1", "agrid2", "bgrid1", "bgrid2",
    "a11", "a12", "a21", "a22",
]
EDGE_NAMES = ["edge_w", "edge_e", "edge_s", "edge_n"]


def bind():
    """The FP64 library with fv3b_generate_grid's argument types set (the
    generator writes FP64 in both builds)."""
    L = _lib.lib("f64")
    L.fv3b_generate_grid.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.POINTER(GridFields), ctypes.c_void_p]
    L.fv3b_generate_grid.restype = ctypes.c_int
    return L


class GridFields(ctypes.Structure):
    _fields_ = [("field", ctypes.c_void_p * len(GRID_FIELD_NAMES)), ("edge", ctypes.c_void_p * 4),
                ("a2b_extrap", ctypes.c_void_p), ("scalars", ctypes.c_void_p)]


class DeviceGrid:
    """Metric terms of an n x n cube (halo ``halo``) generated on ``device``,
    on the equiangular lattice or the reference's gnomonic_ed one
    (``lattice``, as for ``CubedSphereGrid``).

    Attributes: the 2-D fields of ``GRID_FIELD_NAMES`` ([6, m, m] FP64 tensors
    indexed [tile, j, i], m = n + 2 halo + 1), ``edge_w`` .. ``edge_n``,
    ``a2b_extrap``, and the floats ``da_min``, ``da_max``, ``da_min_c``,
    ``da_max_c``.  ``layout`` is ``"ji"``: ``GridData`` uses the tensors as
    they are."""

    layout = "ji"

    def __init__(self, n, halo=3, radius=constants.RADIUS, omega=constants.OMEGA, device="cuda",
                 lattice="equiangular"):
        if lattice not in LATTICES:
            raise ValueError(f"lattice must be one of {LATTICES}, got {lattice!r}")
        self.n, self.halo, self.radius, self.lattice = int(n), int(halo), float(radius), lattice
        m = self.n + 2 * self.halo + 1
        dev = torch.device(device)
        kw = dict(dtype=torch.float64, device=dev)
        out = GridFields()
        for k, name in enumerate(GRID_FIELD_NAMES):
            t = torch.empty((6, m, m), **kw)
            setattr(self, name, t)
            out.field[k] = t.data_ptr()
        for e, name in enumerate(EDGE_NAMES):
            t = torch.empty((6, self.n + 1), **kw)
            setattr(self, name, t)
            out.edge[e] = t.data_ptr()
        self.a2b_extrap = torch.empty((6, 4, 3), **kw)
        scalars = torch.empty(4, **kw)
        out.a2b_extrap = self.a2b_extrap.data_ptr()
        out.scalars = scalars.data_ptr()
        L = bind()
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream().cuda_stream
            rc = L.fv3b_generate_grid(self.n, self.halo, LATTICES.index(lattice), self.radius, float(omega),
                                      ctypes.byref(out), ctypes.c_void_p(stream))
            if rc != 0:
                raise RuntimeError(f"fv3b_generate_grid failed ({rc}): {L.fv3b_last_error().decode()}")
            self.da_min, self.da_max, self.da_min_c, self.da_max_c = (float(v) for v in scalars.cpu())
