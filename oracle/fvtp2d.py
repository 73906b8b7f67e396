"""Finite-volume transport (reference ``fv3core/stencils/fvtp2d.py``) and
del-n flux damping (``fv3core/stencils/delnflux.py``).

Per-level namelist columns (nord, damping) are 1-D arrays indexed by k; the
reference folds them into four vertical bands (k = 0, 1, 2 and 3+) through
compile-time externals nord0..nord3 (delnflux.py:1078-1083), restated here
by ``_band``.
"""
import numpy as np

from . import corners
from ._util import Tile, c3, put, sh
from .ppm import ppm_flux


def _band(col, k):
    """Value of a 4-band column parameter at level k (delnflux.py intervals)."""
    return col[min(k, 3)]


def copy_corners_xy(t: Tile, q, y_field, nk):
    """CopyCornersXY (corners.py:64-117) on dims (X, Y, Z_INTERFACE): q is
    overwritten in place with its x-differenceable copy; returns the
    y-differenceable copy written into ``y_field``."""
    full = t.m - 1
    qx = corners.copy_corners(t, q, "x")
    qy = corners.copy_corners(t, q, "y")
    put(y_field, qy, 0, full, 0, full, 0, nk)
    put(q, qx, 0, full, 0, full, 0, nk)
    return q, y_field


class FvTp2dScratch:
    """Storages a FiniteVolumeTransport instance keeps between calls
    (fvtp2d.py:170-183); NaN until first written."""

    def __init__(self, shape):
        self.q_y_advected_mean = np.full(shape, np.nan)
        self.q_x_advected_mean = np.full(shape, np.nan)
        self.q_advected_y = np.full(shape, np.nan)
        self.q_advected_x = np.full(shape, np.nan)
        self.q_advected_y_x_advected_mean = np.full(shape, np.nan)
        self.q_advected_x_y_advected_mean = np.full(shape, np.nan)


def fvtp2d(t: Tile, g, q_base, q_x, q_y, crx, cry, xfx, yfx, fx_out, fy_out, hord, scratch,
           x_mass_flux=None, y_mass_flux=None, mass=None, nord=None, damp_c=None, deln_scratch=None):
    """FiniteVolumeTransport.__call__ (fvtp2d.py:249-362).  q_x/q_y are the
    corner-copied x/y-differenceable versions of q; outputs fx_out/fy_out."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    nk = t.nz + 1
    area = c3(g.area)
    ord_in = 8 if hord == 10 else hord
    S = scratch
    # y_piecewise_parabolic_inner: i in [is-3, ie+4], j in [js, je+1]
    put(S.q_y_advected_mean, ppm_flux(t, q_y, cry, g.dya, 1, ord_in), s - 3, e + 5, js, je + 2, 0, nk)
    # q_i_stencil (fvtp2d.py:33-47): i in [0, n+6), j in [js, je+4)
    fyy = yfx * S.q_y_advected_mean
    qi = (q_y * area + fyy - sh(fyy, 0, 1)) / (area + yfx - sh(yfx, 0, 1))
    put(S.q_advected_y, qi, 0, t.m - 1, js, je + 4, 0, nk)
    # x_piecewise_parabolic_outer: i in [is, ie+1], j in [js, je+1]
    put(S.q_advected_y_x_advected_mean, ppm_flux(t, S.q_advected_y, crx, g.dxa, 0, hord), s, e + 2, js, je + 2, 0, nk)
    # x_piecewise_parabolic_inner: i in [is, ie+1], j in [js-3, je+4]
    put(S.q_x_advected_mean, ppm_flux(t, q_x, crx, g.dxa, 0, ord_in), s, e + 2, js - 3, je + 5, 0, nk)
    # q_j_stencil (fvtp2d.py:50-60): i in [is, ie+4), j in [0, n+6)
    fx1 = xfx * S.q_x_advected_mean
    awx = area + xfx - sh(xfx, 1, 0)
    qj = (q_x * area + fx1 - sh(fx1, 1, 0)) / awx
    put(S.q_advected_x, qj, s, e + 4, 0, t.m - 1, 0, nk)
    # y_piecewise_parabolic_outer
    put(S.q_advected_x_y_advected_mean, ppm_flux(t, S.q_advected_x, cry, g.dya, 1, hord), s, e + 2, js, je + 2, 0, nk)
    # final_fluxes (fvtp2d.py:63-93)
    xu = xfx if x_mass_flux is None else x_mass_flux
    yu = yfx if y_mass_flux is None else y_mass_flux
    xf = 0.5 * (S.q_advected_y_x_advected_mean + S.q_x_advected_mean) * xu
    yf = 0.5 * (S.q_advected_x_y_advected_mean + S.q_y_advected_mean) * yu
    put(fx_out, xf, s, e + 2, js, je + 1, 0, nk)
    put(fy_out, yf, s, e + 1, js, je + 2, 0, nk)
    if nord is not None and damp_c is not None:
        delnflux(t, g, q_base, fx_out, fy_out, nord, damp_c, deln_scratch, mass=mass)


def calc_damp(nord, damp_c, da_min, nk):
    """delnflux.py:24-26 (FORWARD over the column)."""
    return np.array([(damp_c[k] * da_min) ** (nord[k] + 1) for k in range(nk)])


class DelnScratch:
    def __init__(self, shape, d2_shape=None):
        self.fx2 = np.full(shape, np.nan)
        self.fy2 = np.full(shape, np.nan)
        self.d2 = np.full(d2_shape or shape, np.nan)


def delnflux(t: Tile, g, q, fx, fy, nord, damp_c, scr, mass=None):
    """DelnFlux.__call__ (delnflux.py:963-998)."""
    nz = t.nz
    if np.all(np.asarray(damp_c) <= 1e-4):
        return
    if np.any(np.asarray(damp_c)[:-1] <= 1e-4):
        raise NotImplementedError("damp_c currently must be always greater than 10^-4 for delnflux")
    damp = calc_damp(nord, damp_c, g.da_min, nz)
    delnflux_nosg(t, g, q, scr.fx2, scr.fy2, damp, scr.d2, nord, mass=mass, nk=nz)
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    dk = damp[None, None, :]
    if mass is None:
        fxn = fx[:, :, :nz] + scr.fx2[:, :, :nz]
        fyn = fy[:, :, :nz] + scr.fy2[:, :, :nz]
    else:
        fxn = fx[:, :, :nz] + 0.5 * dk * (sh(mass, -1, 0)[:, :, :nz] + mass[:, :, :nz]) * scr.fx2[:, :, :nz]
        fyn = fy[:, :, :nz] + 0.5 * dk * (sh(mass, 0, -1)[:, :, :nz] + mass[:, :, :nz]) * scr.fy2[:, :, :nz]
    fx[s : e + 2, js : je + 2, :nz] = fxn[s : e + 2, js : je + 2]
    fy[s : e + 2, js : je + 2, :nz] = fyn[s : e + 2, js : je + 2]


def _put_band(dst, val, nord, nk, box_any, box_zero):
    """Store val per level: levels whose band nord is 0 use box_zero, others
    box_any (boxes are (i0, i1, j0, j1), absolute, half open)."""
    for k in range(nk):
        b = box_zero if _band(nord, k) == 0 else box_any
        if b is None:
            continue
        i0, i1, j0, j1 = b
        dst[i0:i1, j0:j1, k] = val[i0:i1, j0:j1, k]


def _copy_corners_nord(t, d2, nord, nk, direction):
    """copy_corners_{x,y}_nord (delnflux.py:297-899): corner copies only on
    levels whose band nord > 0."""
    full = t.m - 1
    res = corners.copy_corners(t, d2, direction)
    for k in range(nk):
        if _band(nord, k) > 0:
            d2[:full, :full, k] = res[:full, :full, k]


def delnflux_nosg(t: Tile, g, q, fx2, fy2, damp, d2, nord, mass=None, nk=None):
    """DelnFluxNoSG.__call__ (delnflux.py:1156-1207)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    if nk is None:
        nk = t.nz
    nmax = int(max(nord))
    if nmax > 3:
        raise ValueError("nord must be less than 3")
    if nk <= 3:
        raise NotImplementedError("nk must be more than 3 for DelnFluxNoSG")
    del6_u, del6_v, rarea = c3(g.del6_u), c3(g.del6_v), c3(g.rarea)
    # d2_damp_interval / copy_stencil_interval
    box_d2 = (s - 1 - nmax, e + 2 + nmax, js - 1 - nmax, je + 2 + nmax)
    box_d2_0 = (s - 1, e + 2, js - 1, je + 2)
    if mass is None:
        val = np.asarray(damp)[None, None, :nk] * q[:, :, :nk]
    else:
        val = q[:, :, :nk]
    _put_band(d2, val, nord, nk, box_d2, box_d2_0)
    _copy_corners_nord(t, d2, nord, nk, "x")
    fx = del6_v * (sh(d2, -1, 0) - d2)
    _put_band(fx2, fx, nord, nk, (s - nmax, e + 2 + nmax, js - nmax, je + 1 + nmax), (s, e + 2, js, je + 1))
    _copy_corners_nord(t, d2, nord, nk, "y")
    fy = del6_u * (sh(d2, 0, -1) - d2)
    _put_band(fy2, fy, nord, nk, (s - nmax, e + 1 + nmax, js - nmax, je + 2 + nmax), (s, e + 1, js, je + 2))
    for n in range(nmax):
        nt = nmax - 1 - n
        val = (fx2 - sh(fx2, 1, 0) + fy2 - sh(fy2, 0, 1)) * rarea
        _put_band(d2, val, nord, nk, (s - nt - 1, e + nt + 2, js - nt - 1, je + nt + 2), None)
        _copy_corners_nord(t, d2, nord, nk, "x")
        fx = -del6_v * (sh(d2, -1, 0) - d2)
        _put_band(fx2, fx, nord, nk, (s - nt, e + nt + 2, js - nt, je + nt + 1), None)
        _copy_corners_nord(t, d2, nord, nk, "y")
        fy = -del6_u * (sh(d2, 0, -1) - d2)
        _put_band(fy2, fy, nord, nk, (s - nt, e + nt + 1, js - nt, je + nt + 2), None)
