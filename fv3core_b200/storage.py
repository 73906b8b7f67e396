"""Device storage for the six-tile fields.

A field lives on the GPU as one contiguous torch tensor in the kernel layout
``[6, nk, nj, ni]`` (i fastest).  ``as_reference_view`` returns the
``[6, ni, nj, nk]`` view that matches the reference's (i, j, k) indexing, so
host code can index fields exactly like gt4py storages; the view shares
memory with the kernel layout.
"""
import numpy as np
import torch

from ._lib import GridDims


class GridIndexing:
    """Index helper with the reference's names (fv3core/utils/stencil.py:280-642)
    for all six tiles of an n x n x npz cube."""

    def __init__(self, domain, n_halo=3, south_edge=True, north_edge=True, west_edge=True, east_edge=True,
                 precision="f64", members=1):
        self.domain = tuple(int(x) for x in domain)
        # cubes held in every array: 1, or the members of a batched ensemble
        # (member m owns tile slots 6m .. 6m+5)
        self.members = int(members)
        self.n_halo = int(n_halo)
        if self.domain[0] != self.domain[1]:
            raise ValueError("cube tiles must be square")
        if not (south_edge and north_edge and west_edge and east_edge):
            raise NotImplementedError("each device array holds whole tiles (layout 1x1)")
        self.origin = (self.n_halo, self.n_halo, 0)
        # the device context (fv3b_ctx*) of the GridData built on this grid;
        # every stage class reaches the metric terms and workspace through it
        self.context = None
        # "f64" (FP64 fields) or "f32" (the mixed-precision build's FP32 fields)
        self.precision = precision

    @property
    def ntiles(self):
        return 6 * self.members

    @property
    def dtype(self):
        return torch.float32 if self.precision == "f32" else torch.float64

    @property
    def n(self):
        return self.domain[0]

    @property
    def npz(self):
        return self.domain[2]

    @property
    def isc(self):
        return self.n_halo

    @property
    def iec(self):
        return self.n_halo + self.n - 1

    jsc = isc
    jec = iec

    @property
    def max_shape(self):
        m = self.n + 2 * self.n_halo + 1
        return (m, m, self.npz + 1)

    def dims(self):
        return GridDims(self.n, self.n_halo, self.npz, 0)


def empty(gi: GridIndexing, kind="3d", device="cuda", dtype=None):
    m, _, nk = gi.max_shape
    dtype = gi.dtype if dtype is None else dtype
    nt = gi.ntiles
    if kind == "3d":
        t = torch.empty((nt, nk, m, m), device=device, dtype=dtype)
    elif kind == "2d":
        t = torch.empty((nt, m, m), device=device, dtype=dtype)
    elif kind == "1d":
        t = torch.empty((nk,), device=device, dtype=dtype)
    else:
        raise ValueError(kind)
    return t


def zeros(gi, kind="3d", device="cuda", dtype=None):
    return empty(gi, kind, device, dtype).zero_()


def to_device(a: np.ndarray, device="cuda", dtype=torch.float64):
    """numpy [6, i, j, k] (or [6, i, j], or [k]) -> device kernel layout."""
    a = np.asarray(a)
    if a.ndim == 4:
        a = np.ascontiguousarray(a.transpose(0, 3, 2, 1))
    elif a.ndim == 3:
        a = np.ascontiguousarray(a.transpose(0, 2, 1))
    return torch.from_numpy(a).to(device=device, dtype=dtype)


def to_host(t: torch.Tensor) -> np.ndarray:
    """device kernel layout -> numpy [6, i, j, k] / [6, i, j] / [k]."""
    a = t.detach().to("cpu", torch.float64).numpy()
    if a.ndim == 4:
        return np.ascontiguousarray(a.transpose(0, 3, 2, 1))
    if a.ndim == 3:
        return np.ascontiguousarray(a.transpose(0, 2, 1))
    return a.copy()


def as_reference_view(t: torch.Tensor) -> torch.Tensor:
    if t.dim() == 4:
        return t.permute(0, 3, 2, 1)
    if t.dim() == 3:
        return t.permute(0, 2, 1)
    return t


def check_field(t, gi, kind, name):
    m, _, nk = gi.max_shape
    nt = gi.ntiles
    want = {"3d": (nt, nk, m, m), "2d": (nt, m, m), "1d": (nk,)}[kind]
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch tensor in device layout, got {type(t).__name__}")
    if tuple(t.shape) != want or not t.is_contiguous():
        raise ValueError(f"{name}: expected contiguous device layout {want}, got {tuple(t.shape)}")
    if t.dtype != gi.dtype:
        raise TypeError(f"{name}: expected {gi.dtype}, got {t.dtype}")
    if not t.is_cuda:
        raise ValueError(f"{name}: must be a CUDA tensor")
    return t.data_ptr()


def stream_ptr():
    return torch.cuda.current_stream().cuda_stream
