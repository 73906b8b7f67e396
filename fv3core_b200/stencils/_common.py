"""Helpers shared by the stage classes."""
import numpy as np
import torch

from ..storage import check_field


def context(stencil_factory):
    ctx = stencil_factory.grid_indexing.context
    if ctx is None:
        raise RuntimeError(
            "no device context on this grid: build a fv3core_b200.grid_data.GridData for the "
            "StencilFactory's grid_indexing first"
        )
    return ctx


def host_column(a, n, name):
    """A K field (the reference's FloatFieldK) as a contiguous host float64
    array of at least n values."""
    if isinstance(a, torch.Tensor):
        a = a.detach().to("cpu", torch.float64).numpy()
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if a.ndim != 1 or a.shape[0] < n:
        raise ValueError(f"{name}: expected a 1-D array of at least {n} values, got shape {a.shape}")
    return a


def ptrs(gi, kind, **fields):
    return [check_field(t, gi, kind, name) for name, t in fields.items()]
