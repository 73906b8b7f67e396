"""numpy-backed storages with the gt4py v36 constructor signatures."""
import numpy as np

from . import storage  # noqa: F401
from .storage import Storage


def _shape_for(shape, mask):
    shape = tuple(int(s) for s in shape)
    if mask is None:
        return shape
    n_true = sum(1 for m in mask if m)
    if len(shape) == n_true:
        return shape
    if len(shape) == len(mask):
        return tuple(s for s, m in zip(shape, mask) if m)
    return shape


def _make(data, default_origin, mask):
    st = np.asarray(data, dtype=np.float64 if data.dtype.kind == "f" else data.dtype).view(Storage)
    st.default_origin = tuple(default_origin) if default_origin is not None else None
    st.mask = mask
    return st


def empty(backend=None, default_origin=None, shape=None, dtype=np.float64, mask=None, managed_memory=True, **kw):
    # uninitialised memory is modelled as NaN so that any read of it is visible
    data = np.full(_shape_for(shape, mask), np.nan, dtype=dtype)
    return _make(data, default_origin, mask)


def zeros(backend=None, default_origin=None, shape=None, dtype=np.float64, mask=None, managed_memory=True, **kw):
    data = np.zeros(_shape_for(shape, mask), dtype=dtype)
    return _make(data, default_origin, mask)


def ones(backend=None, default_origin=None, shape=None, dtype=np.float64, mask=None, managed_memory=True, **kw):
    data = np.ones(_shape_for(shape, mask), dtype=dtype)
    return _make(data, default_origin, mask)


def from_array(data, backend=None, default_origin=None, shape=None, dtype=np.float64, mask=None, managed_memory=True, **kw):
    arr = np.array(np.asarray(data), dtype=dtype, copy=True)
    if shape is not None:
        tgt = _shape_for(shape, mask)
        if arr.shape != tgt and arr.size == int(np.prod(tgt)):
            arr = arr.reshape(tgt)
    return _make(arr, default_origin, mask)
