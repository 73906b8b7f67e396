"""Device-resident grid metrics and the C-ABI context.

``GridData`` plays the role of the reference's ``GridData`` +
``DampingCoefficients`` (fv3core/utils/grid.py:475-799): it holds the 2-D
metric fields, here uploaded once to the GPU for all six tiles, and owns the
``fv3b_ctx`` (metric pointers + device workspace) that every stage call uses.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .grid import CubedSphereGrid
from .storage import GridIndexing

METRIC_FIELDS = [
    "dx", "dy", "dxa", "dya", "dxc", "dyc",
    "rdx", "rdy", "rdxa", "rdya", "rdxc", "rdyc",
    "area", "rarea", "rarea_c",
    "sin_sg1", "sin_sg2", "sin_sg3", "sin_sg4",
    "cos_sg1", "cos_sg2", "cos_sg3", "cos_sg4",
    "cosa", "cosa_u", "cosa_v", "cosa_s", "sina_u", "sina_v",
    "rsina", "rsin_u", "rsin_v", "rsin2",
    "del6_u", "del6_v", "divg_u", "divg_v",
    "fC", "f0",
    "agrid1", "agrid2", "bgrid1", "bgrid2",
    "edge_w", "edge_e", "edge_s", "edge_n",
    "a2b_extrap",
]
# 2-D fields on the device that are not part of the C ABI's metric struct:
# the cubed-to-latlon coefficients (the reference keeps them on its legacy
# grid, not in GridData), passed to fv3b_cubed_to_latlon directly
EXTRA_FIELDS = ["a11", "a12", "a21", "a22"]


class Metrics(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in METRIC_FIELDS] + [
        ("da_min", ctypes.c_double),
        ("da_min_c", ctypes.c_double),
    ]



class GridData:
    """All metric terms of an n x n cube on the GPU, plus the stage context.

    ``members`` > 1 makes the context of an ensemble of that many cubes of
    this grid advanced together (fv3b_ctx_create_batched): every field then
    holds 6 x members tile slots, and the metric terms are repeated for each
    member."""

    def __init__(self, grid: CubedSphereGrid, npz: int, device="cuda", precision="f64", members=1):
        self.grid = grid
        self.precision = precision
        self.members = int(members)
        self.grid_indexing = GridIndexing((grid.n, grid.n, npz), grid.halo, precision=precision,
                                          members=self.members)
        tdtype = self.grid_indexing.dtype
        self.device = device
        self.tensors = {}
        for name in METRIC_FIELDS + EXTRA_FIELDS:
            if getattr(grid, "layout", "ij") == "ji":
                # generated on the device (grid_device.DeviceGrid): FP64
                # tensors already in the kernels' layout
                t = getattr(grid, name).to(device=device, dtype=tdtype)
                if self.members > 1:
                    t = t.repeat(self.members, *([1] * (t.dim() - 1)))
                self.tensors[name] = t.contiguous()
                setattr(self, name, self.tensors[name])
                continue
            a = np.asarray(getattr(grid, name), dtype=np.float64)
            if self.members > 1:  # the same metric terms for every member
                a = np.concatenate([a] * self.members, axis=0)
            if a.ndim == 3 and name != "a2b_extrap":  # [6, i, j] -> [6, j, i]
                t = torch.from_numpy(np.ascontiguousarray(a.transpose(0, 2, 1))).to(device=device, dtype=tdtype)
            else:  # edge factors [6, n+1], corner ratios [6, 4, 3]
                t = torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=tdtype)
            self.tensors[name] = t
            setattr(self, name, t)
        self.da_min = grid.da_min
        self.da_min_c = grid.da_min_c
        m = Metrics()
        for name in METRIC_FIELDS:
            setattr(m, name, self.tensors[name].data_ptr())
        m.da_min = self.da_min
        m.da_min_c = self.da_min_c
        self._metrics = m
        self._dims = self.grid_indexing.dims()
        L = _lib.lib(precision)
        L.fv3b_ctx_create_batched.argtypes = [ctypes.POINTER(_lib.GridDims), ctypes.POINTER(Metrics), ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_void_p)]
        L.fv3b_ctx_create_batched.restype = ctypes.c_int
        L.fv3b_ctx_destroy.argtypes = [ctypes.c_void_p]
        L.fv3b_ctx_destroy.restype = ctypes.c_int
        ctx = ctypes.c_void_p()
        rc = L.fv3b_ctx_create_batched(ctypes.byref(self._dims), ctypes.byref(m), self.members, ctypes.byref(ctx))
        if rc != 0:
            raise RuntimeError(f"fv3b_ctx_create failed ({rc}): {L.fv3b_last_error().decode()}")
        self.ctx = ctx
        _lib.register_context(ctx, precision)
        self.grid_indexing.context = ctx

    def close(self):
        if getattr(self, "ctx", None) is not None and self.ctx.value:
            _lib.lib(self.precision).fv3b_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
