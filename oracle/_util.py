"""numpy helpers for the oracle: shifted reads, region masks, box writes.

Arrays are one tile's storages ``[m, m, nk]`` (3-D) or ``[m, m]`` (2-D); 2-D
metric arrays are used as ``[m, m, 1]`` so that they broadcast over k.
"""
import numpy as np


class Tile:
    """Index set of one tile (reference GridIndexing with all four edges)."""

    def __init__(self, n, nz, h=3):
        self.n, self.nz, self.h = n, nz, h
        self.isc = self.jsc = h
        self.iec = self.jec = h + n - 1
        self.m = n + 2 * h + 1
        self.nk = nz + 1


def c3(a):
    """2-D metric -> [m, m, 1] for broadcasting."""
    a = np.asarray(a, dtype=np.float64)
    return a[:, :, None] if a.ndim == 2 else a


def sh(a, di=0, dj=0, dk=0):
    """b[i, j, k] = a[i+di, j+dj, k+dk] (NaN where that leaves the array)."""
    a = c3(a)
    out = np.full(a.shape, np.nan)
    src = []
    dst = []
    for d, n in zip((di, dj, dk), a.shape):
        if d >= 0:
            src.append(slice(d, n))
            dst.append(slice(0, n - d))
        else:
            src.append(slice(0, n + d))
            dst.append(slice(-d, n))
    if a.shape[2] == 1 and dk != 0:
        raise ValueError("vertical shift of a 2-D field")
    out[tuple(dst)] = a[tuple(src)]
    return out


def region(t: Tile, i0=None, i1=None, j0=None, j1=None):
    """Boolean [m, m, 1] mask of absolute storage indices i0 <= i < i1,
    j0 <= j < j1 (None = unbounded)."""
    m = np.zeros((t.m, t.m, 1), dtype=bool)
    a0 = 0 if i0 is None else max(i0, 0)
    a1 = t.m if i1 is None else min(i1, t.m)
    b0 = 0 if j0 is None else max(j0, 0)
    b1 = t.m if j1 is None else min(j1, t.m)
    if a1 > a0 and b1 > b0:
        m[a0:a1, b0:b1] = True
    return m


def at(t: Tile, i=None, j=None):
    """Mask of a single column i and/or row j (None = all)."""
    return region(t, i, None if i is None else i + 1, j, None if j is None else j + 1)


def put(dst, val, i0, i1, j0, j1, k0=0, k1=None, mask=None):
    """dst[i0:i1, j0:j1, k0:k1] = val over that box, where ``mask`` (full
    array shaped or broadcastable) is true; val is full-array shaped."""
    if k1 is None:
        k1 = dst.shape[2]
    box = (slice(i0, i1), slice(j0, j1), slice(k0, k1))
    v = np.broadcast_to(val, dst.shape)[box]
    if mask is None:
        dst[box] = v
    else:
        mk = np.broadcast_to(mask, dst.shape)[box]
        dst[box] = np.where(mk, v, dst[box])


def where(mask, a, b):
    return np.where(mask, a, b)
