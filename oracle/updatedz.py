"""Height updates on the C grid (reference ``fv3core/stencils/updatedzc.py``)
and D grid (``fv3core/stencils/updatedzd.py``)."""
import numpy as np

from fv3core_b200 import constants as C

from . import corners
from ._util import Tile, c3, put, sh
from .fvtp2d import FvTp2dScratch, copy_corners_xy, delnflux_nosg, fvtp2d


def update_dz_c(t: Tile, g, dp_ref, zs, ut, vt, gz, ws, dt):
    """UpdateGeopotentialHeightOnCGrid.__call__ (updatedzc.py:123-163):
    gz (interfaces) advected by ut/vt over dt with a DZ_MIN floor; ws at the
    surface.  gz, ws updated in place."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    nz, nk = t.nz, t.nk
    full = t.m - 1
    # double_copy + fill_corners_2cells_{x,y} (updatedzc.py:37-43, 151-156)
    gz_x = np.full(gz.shape, np.nan)
    gz_y = np.full(gz.shape, np.nan)
    put(gz_x, gz, 0, full, 0, full, 0, nk)
    put(gz_y, gz, 0, full, 0, full, 0, nk)
    put(gz_x, corners.fill_corners_2cells_x(t, gz_x), 0, full, 0, full, 0, nk)
    put(gz_y, corners.fill_corners_2cells_y(t, gz_y), 0, full, 0, full, 0, nk)
    dp0 = np.asarray(dp_ref)
    xfx = np.full(gz.shape, np.nan)
    yfx = np.full(gz.shape, np.nan)
    # p_weighted_average_top / domain / bottom (updatedzc.py:15-34)
    ratio = dp0[0] / (dp0[0] + dp0[1])
    xfx[:, :, 0] = ut[:, :, 0] + (ut[:, :, 0] - ut[:, :, 1]) * ratio
    yfx[:, :, 0] = vt[:, :, 0] + (vt[:, :, 0] - vt[:, :, 1]) * ratio
    for k in range(1, nk - 1):
        ir = 1.0 / (dp0[k - 1] + dp0[k])
        xfx[:, :, k] = (dp0[k] * ut[:, :, k - 1] + dp0[k - 1] * ut[:, :, k]) * ir
        yfx[:, :, k] = (dp0[k] * vt[:, :, k - 1] + dp0[k - 1] * vt[:, :, k]) * ir
    k = nk - 1
    ratio = dp0[k - 1] / (dp0[k - 2] + dp0[k - 1])
    xfx[:, :, k] = ut[:, :, k - 1] + (ut[:, :, k - 1] - ut[:, :, k - 2]) * ratio
    yfx[:, :, k] = vt[:, :, k - 1] + (vt[:, :, k - 1] - vt[:, :, k - 2]) * ratio
    fx = xfx * np.where(xfx > 0.0, sh(gz_x, -1, 0), gz_x)
    fy = yfx * np.where(yfx > 0.0, sh(gz_y, 0, -1), gz_y)
    area = c3(g.area)
    new = (gz_y * area + fx - sh(fx, 1, 0) + fy - sh(fy, 0, 1)) / (area + xfx - sh(xfx, 1, 0) + yfx - sh(yfx, 0, 1))
    b = (s - 1, e + 2, js - 1, je + 2)
    put(gz, new, *b, 0, nk)
    rdt = 1.0 / dt
    ws[b[0] : b[1], b[2] : b[3]] = (zs[b[0] : b[1], b[2] : b[3]] - gz[b[0] : b[1], b[2] : b[3], nk - 1]) * rdt
    for k in range(nk - 2, -1, -1):
        v = gz[b[0] : b[1], b[2] : b[3], k]
        kp1 = gz[b[0] : b[1], b[2] : b[3], k + 1] + C.DZ_MIN
        gz[b[0] : b[1], b[2] : b[3], k] = np.where(v > kp1, v, kp1)


def spline_constants(dp0, nk):
    """cubic_spline_interpolation_constants (updatedzd.py:121-145)."""
    gk = np.full(nk, np.nan)
    beta = np.full(nk, np.nan)
    gamma = np.full(nk, np.nan)
    gk[0] = dp0[1] / dp0[0]
    beta[0] = gk[0] * (gk[0] + 0.5)
    gamma[0] = (1.0 + gk[0] * (gk[0] + 1.5)) / beta[0]
    for k in range(1, nk - 1):
        gk[k] = dp0[k - 1] / dp0[k]
        beta[k] = 2.0 + 2.0 * gk[k] - gamma[k - 1]
        gamma[k] = gk[k] / beta[k]
    return gk, beta, gamma


def interpolate_to_interfaces(t: Tile, qc, qi, gk, beta, gamma):
    """cubic_spline_interpolation_from_layer_center_to_interfaces
    (updatedzd.py:148-186) over the full halo domain, levels 0..npz."""
    nk = t.nk
    full = t.m - 1
    S = (slice(0, full), slice(0, full))
    q = qc[S]
    out = qi[S]
    xt1 = 2.0 * gk[0] * (gk[0] + 1.0)
    out[:, :, 0] = (xt1 * q[:, :, 0] + q[:, :, 1]) / beta[0]
    for k in range(1, nk - 1):
        out[:, :, k] = (3.0 * (q[:, :, k - 1] + gk[k] * q[:, :, k]) - out[:, :, k - 1]) / beta[k]
    k = nk - 1
    a_bot = 1.0 + gk[k - 1] * (gk[k - 1] + 1.5)
    xt1 = 2.0 * gk[k - 1] * (gk[k - 1] + 1.0)
    xt2 = gk[k - 1] * (gk[k - 1] + 0.5) - a_bot * gamma[k - 1]
    out[:, :, k] = (xt1 * q[:, :, k - 1] + q[:, :, k - 2] - a_bot * out[:, :, k - 1]) / xt2
    for k in range(nk - 2, -1, -1):
        out[:, :, k] = out[:, :, k] - gamma[k] * out[:, :, k + 1]


class UpdateDzDState:
    def __init__(self, t: Tile, dp0, col):
        shp = (t.m, t.m, t.nk)
        nan = lambda: np.full(shp, np.nan)  # noqa: E731
        self.crx_i, self.cry_i, self.xfx_i, self.yfx_i = nan(), nan(), nan(), nan()
        self.wk, self.gzx_diff, self.gzy_diff, self.fx, self.fy = nan(), nan(), nan(), nan(), nan()
        self.y_temporary = nan()
        self.fvtp = FvTp2dScratch(shp)
        self.gk, self.beta, self.gamma = spline_constants(np.asarray(dp0), t.nk)
        self.col = col
        if any(col["damp_vt"][k] <= 1e-5 for k in range(4)):
            raise NotImplementedError("damp <= 1e-5 in column_cols is untested")


def update_dz_d(t: Tile, g, st: UpdateDzDState, hord_tm, zs, zh, crx, cry, xfx, yfx, wsd, dt):
    """UpdateHeightOnDGrid.__call__ (updatedzd.py:323-393)."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    nk = t.nk
    interpolate_to_interfaces(t, crx, st.crx_i, st.gk, st.beta, st.gamma)
    interpolate_to_interfaces(t, xfx, st.xfx_i, st.gk, st.beta, st.gamma)
    interpolate_to_interfaces(t, cry, st.cry_i, st.gk, st.beta, st.gamma)
    interpolate_to_interfaces(t, yfx, st.yfx_i, st.gk, st.beta, st.gamma)
    copy_corners_xy(t, zh, st.y_temporary, nk)
    fvtp2d(t, g, zh, zh, st.y_temporary, st.crx_i, st.cry_i, st.xfx_i, st.yfx_i, st.fx, st.fy, hord_tm, st.fvtp)
    # DelnFluxNoSG with nk = npz + 1 and the raw damp_vt column as damping
    delnflux_nosg(t, g, zh, st.gzx_diff, st.gzy_diff, np.asarray(st.col["damp_vt"]), st.wk, st.col["nord_v"],
                  nk=nk)
    # apply_height_fluxes (updatedzd.py:63-118) on the compute domain
    area = c3(g.area)
    aaf = (area + st.xfx_i - sh(st.xfx_i, 1, 0)) + (area + st.yfx_i - sh(st.yfx_i, 0, 1)) - area
    adv = (zh * area + st.fx - sh(st.fx, 1, 0) + st.fy - sh(st.fy, 0, 1)) / aaf
    diff = (st.gzx_diff - sh(st.gzx_diff, 1, 0) + st.gzy_diff - sh(st.gzy_diff, 0, 1)) / area
    put(zh, adv + diff, s, e + 1, js, je + 1, 0, nk)
    I, J = slice(s, e + 1), slice(js, je + 1)
    wsd[I, J] = (zs[I, J] - zh[I, J, nk - 1]) / dt
    for k in range(nk - 2, -1, -1):
        v = zh[I, J, k]
        other = zh[I, J, k + 1] + C.DZ_MIN
        zh[I, J, k] = np.where(v > other, v, other)
