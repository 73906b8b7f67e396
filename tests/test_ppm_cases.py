"""Hand-constructed PPM cases on the oracle's flux (xppm.py's compute_x_flux
restated in oracle/ppm.py), the reference of the CUDA transport:

* a constant field is transported unchanged: the interface mean is the
  constant for any Courant number;
* on a uniform grid a linear field is reproduced exactly: the interface mean
  is the exact average of the line over the upwind part of the cell;
* a step stays bounded: every interface mean lies between the field's
  extremes (the monotonic limiter, mord = 6)."""
import numpy as np
import pytest

from oracle import ppm
from oracle._util import Tile

N, NZ = 12, 1


def _interior(t, a, axis):
    """Interfaces whose whole stencil lies away from the tile edges."""
    s, e = t.isc + 3, t.iec - 2
    return a[s:e, s:e, 0]


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("c", [-0.7, -0.2, 0.3, 0.9])
def test_constant_field(axis, c):
    t = Tile(N, NZ)
    q = np.full((t.m, t.m, 1), 3.25)
    dxa = np.ones((t.m, t.m))
    f = ppm.ppm_flux(t, q, np.full(q.shape, c), dxa, axis)
    np.testing.assert_allclose(_interior(t, f, axis), 3.25, rtol=0, atol=1e-14)


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("c", [-0.6, 0.4])
def test_linear_field_is_exact(axis, c):
    t = Tile(N, NZ)
    idx = np.arange(t.m, dtype=np.float64)
    line = 2.0 + 0.5 * idx
    q = (line[:, None] if axis == 0 else line[None, :])[:, :, None] * np.ones((t.m, t.m, 1))
    dxa = np.ones((t.m, t.m))
    f = ppm.ppm_flux(t, q, np.full(q.shape, c), dxa, axis)
    # interface i sits between cells i-1 and i; with c > 0 the upwind part
    # is the last c of cell i-1, with c < 0 the first |c| of cell i
    x = idx[:, None] if axis == 0 else idx[None, :]
    exact = (2.0 + 0.5 * (x - 1)) + 0.5 * (1.0 - c) / 2.0 if c > 0 else (2.0 + 0.5 * x) - 0.5 * (1.0 + c) / 2.0
    exact = exact * np.ones((t.m, t.m))
    np.testing.assert_allclose(_interior(t, f, axis), _interior(t, exact[:, :, None], axis), rtol=1e-14)


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("c", [-0.8, 0.5])
def test_step_stays_bounded(axis, c):
    t = Tile(N, NZ)
    idx = np.arange(t.m)
    line = np.where(idx < t.m // 2, 1.0, 5.0)
    q = (line[:, None] if axis == 0 else line[None, :])[:, :, None] * np.ones((t.m, t.m, 1))
    dxa = np.ones((t.m, t.m))
    f = _interior(t, ppm.ppm_flux(t, q, np.full(q.shape, c), dxa, axis), axis)
    assert f.min() >= 1.0 - 1e-14 and f.max() <= 5.0 + 1e-14
