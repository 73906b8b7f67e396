"""C-grid shallow water (reference ``fv3core/stencils/c_sw.py``) with its
D->A->C wind interpolation (``fv3core/stencils/d2a2c_vect.py``).

All functions work on one tile (``Tile``) and a metric namespace ``g`` whose
attributes are that tile's 2-D metric arrays.
"""
import numpy as np

from . import corners
from ._util import Tile, at, c3, put, region, sh

# d2a2c_vect.py:13-15 and a2b_ord4.py:24-35
C1, C2, C3 = -2.0 / 14.0, 11.0 / 14.0, 5.0 / 14.0
A1, A2 = 9.0 / 16.0, -1.0 / 16.0
BIG = 1e30


def contravariant(v1, v2, cosa, rsin2):
    """d2a2c_vect.py:185-236."""
    return (v1 - v2 * cosa) * rsin2


def _edge_interpolate4_x(ua, dxa):
    """d2a2c_vect.py:357-363 (n2 uses t1, as in the reference)."""
    t1 = sh(dxa, -2, 0) + sh(dxa, -1, 0)
    t2 = dxa + sh(dxa, 1, 0)
    n1 = (t1 + sh(dxa, -1, 0)) * sh(ua, -1, 0) - sh(dxa, -1, 0) * sh(ua, -2, 0)
    n2 = (t1 + dxa) * ua - dxa * sh(ua, 1, 0)
    return 0.5 * (n1 / t1 + n2 / t2)


def _edge_interpolate4_y(va, dya):
    """d2a2c_vect.py:366-372."""
    t1 = sh(dya, 0, -2) + sh(dya, 0, -1)
    t2 = dya + sh(dya, 0, 1)
    n1 = (t1 + sh(dya, 0, -1)) * sh(va, 0, -1) - sh(dya, 0, -1) * sh(va, 0, -2)
    n2 = (t1 + dya) * va - dya * sh(va, 0, 1)
    return 0.5 * (n1 / t1 + n2 / t2)


def d2a2c_vect(t: Tile, g, uc, vc, u, v, ua, va, utc, vtc):
    """DGrid2AGrid2CGridVectors.__call__ (d2a2c_vect.py:543-651), dord4=True,
    not nested.  Updates uc, vc, ua, va, utc, vtc in place."""
    nz = t.nz
    s, e = t.isc, t.iec
    n = t.n
    cosa_s, cosa_u, cosa_v = c3(g.cosa_s), c3(g.cosa_u), c3(g.cosa_v)
    rsin_u, rsin_v, rsin2 = c3(g.rsin_u), c3(g.rsin_v), c3(g.rsin2)
    dxa, dya = c3(g.dxa), c3(g.dya)
    sin_sg1, sin_sg2, sin_sg3, sin_sg4 = c3(g.sin_sg1), c3(g.sin_sg2), c3(g.sin_sg3), c3(g.sin_sg4)
    npt = 4
    if npt > n - 1:
        npt = 0
    nx = e + 1
    # set_tmps (d2a2c_vect.py:18-21): full halo domain
    full = t.m - 1
    utmp = np.full(u.shape, np.nan)
    vtmp = np.full(u.shape, np.nan)
    utmp[:full, :full, :nz] = BIG
    vtmp[:full, :full, :nz] = BIG
    lo = npt + 2  # OFFSET = 2
    hi = nx - npt
    # lagrange_interpolation_y_p1 / x_p1 (d2a2c_vect.py:141-161)
    val = A2 * (sh(u, 0, -1) + sh(u, 0, 2)) + A1 * (u + sh(u, 0, 1))
    put(utmp, val, lo, hi + 1, lo, hi + 1, 0, nz)
    val = A2 * (sh(v, -1, 0) + sh(v, 2, 0)) + A1 * (v + sh(v, 1, 0))
    put(vtmp, val, lo, hi + 1, lo, hi + 1, 0, nz)
    # avg_box (d2a2c_vect.py:164-182)
    off = -1 if npt == 0 else 3
    mask = (
        region(t, None, None, None, t.jsc + off)
        | region(t, None, None, t.jec - off + 1, None)
        | region(t, None, s + off, None, None)
        | region(t, e - off + 1, None, None, None)
    )
    put(utmp, 0.5 * (u + sh(u, 0, 1)), 0, full, 0, full, 0, nz, mask)
    put(vtmp, 0.5 * (v + sh(v, 1, 0)), 0, full, 0, full, 0, nz, mask)
    # contravariant_components (d2a2c_vect.py:248-260)
    put(ua, contravariant(utmp, vtmp, cosa_s, rsin2), s - 2, e + 3, s - 2, e + 3, 0, nz)
    put(va, contravariant(vtmp, utmp, cosa_s, rsin2), s - 2, e + 3, s - 2, e + 3, 0, nz)
    # fill_corners_x (d2a2c_vect.py:24-32)
    b0, b1 = s - 3, e + 4
    new_utmp = corners.fill_corners_3cells_mult_x(t, utmp, vtmp, -1.0, 1.0, 1.0, -1.0)
    new_ua = corners.fill_corners_2cells_mult_x(t, ua, va, -1.0, 1.0, 1.0, -1.0)
    put(utmp, new_utmp, b0, b1, b0, b1, 0, nz)
    put(ua, new_ua, b0, b1, b0, b1, 0, nz)
    # ut_main (d2a2c_vect.py:263-273)
    ucv = A2 * (sh(utmp, -2, 0) + sh(utmp, 1, 0)) + A1 * (sh(utmp, -1, 0) + utmp)
    put(uc, ucv, s + 2, e, t.jsc - 1, t.jec + 2, 0, nz)
    put(utc, contravariant(uc, v, cosa_u, rsin_u), s + 2, e, t.jsc - 1, t.jec + 2, 0, nz)
    # east_west_edges (d2a2c_vect.py:45-93), rows js-1 .. je+1
    J0, J1 = t.jsc - 1, t.jec + 2

    def col(i):
        return region(t, i, i + 1, J0, J1)

    vol_x = C1 * sh(utmp, -2, 0) + C2 * sh(utmp, -1, 0) + C3 * utmp
    vol_x_rev = C1 * sh(utmp, 1, 0) + C2 * utmp + C3 * sh(utmp, -1, 0)
    e4 = _edge_interpolate4_x(ua, dxa)
    for (im1, i0, ip1) in ((s - 1, s, s + 1), (e, e + 1, e + 2)):
        put(uc, vol_x, b0, b1, b0, b1, 0, nz, col(im1))
        put(utc, e4, b0, b1, b0, b1, 0, nz, col(i0))
        ucv = np.where(utc > 0, utc * sh(sin_sg3, -1, 0), utc * sin_sg1)
        put(uc, ucv, b0, b1, b0, b1, 0, nz, col(i0))
        put(uc, vol_x_rev, b0, b1, b0, b1, 0, nz, col(ip1))
        put(utc, contravariant(uc, v, cosa_u, rsin_u), b0, b1, b0, b1, 0, nz, col(im1))
        put(utc, contravariant(uc, v, cosa_u, rsin_u), b0, b1, b0, b1, 0, nz, col(ip1))
    # fill_corners_y (d2a2c_vect.py:35-42)
    new_vtmp = corners.fill_corners_3cells_mult_y(t, vtmp, utmp, -1.0, 1.0, 1.0, -1.0)
    new_va = corners.fill_corners_2cells_mult_y(t, va, ua, -1.0, 1.0, 1.0, -1.0)
    put(vtmp, new_vtmp, b0, b1, b0, b1, 0, nz)
    put(va, new_va, b0, b1, b0, b1, 0, nz)
    # north_south_edges (d2a2c_vect.py:96-138), columns is-1 .. ie+1
    I0, I1 = s - 1, e + 2

    def row(j0, j1=None):
        return region(t, I0, I1, j0, j0 + 1 if j1 is None else j1)

    lag_y = A2 * (sh(vtmp, 0, -2) + sh(vtmp, 0, 1)) + A1 * (sh(vtmp, 0, -1) + vtmp)
    vol_y = C1 * sh(vtmp, 0, -2) + C2 * sh(vtmp, 0, -1) + C3 * vtmp
    vol_y_rev = C1 * sh(vtmp, 0, 1) + C2 * vtmp + C3 * sh(vtmp, 0, -1)
    e4y = _edge_interpolate4_y(va, dya)
    js, je = t.jsc, t.jec
    put(vc, lag_y, b0, b1, b0, b1, 0, nz, row(js - 1, je + 3))
    put(vtc, contravariant(vc, u, cosa_v, rsin_v), b0, b1, b0, b1, 0, nz, row(js - 1, je + 3))
    for (jm1, j0, jp1) in ((js - 1, js, js + 1), (je, je + 1, je + 2)):
        put(vc, vol_y, b0, b1, b0, b1, 0, nz, row(jm1))
        put(vtc, contravariant(vc, u, cosa_v, rsin_v), b0, b1, b0, b1, 0, nz, row(jm1))
        put(vtc, e4y, b0, b1, b0, b1, 0, nz, row(j0))
        vcv = np.where(vtc > 0, vtc * sh(sin_sg4, 0, -1), vtc * sin_sg2)
        put(vc, vcv, b0, b1, b0, b1, 0, nz, row(j0))
        put(vc, vol_y_rev, b0, b1, b0, b1, 0, nz, row(jp1))
        put(vtc, contravariant(vc, u, cosa_v, rsin_v), b0, b1, b0, b1, 0, nz, row(jp1))
    # vt_main (d2a2c_vect.py:276-286)
    put(vc, lag_y, s - 1, e + 2, js + 2, je, 0, nz)
    put(vtc, contravariant(vc, u, cosa_v, rsin_v), s - 1, e + 2, js + 2, je, 0, nz)


def c_sw(t: Tile, g, fC, delp, pt, u, v, w, uc, vc, ua, va, ut, vt, divgd, omga, dt2, nord=3):
    """CGridShallowWaterDynamics.__call__ (c_sw.py:534-659).  Returns
    (delpc, ptc); updates delp/pt/w corner halos, uc, vc, ua, va, ut, vt,
    divgd and omga in place, like the reference."""
    nz = t.nz
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    sin_sg = [None] + [c3(getattr(g, f"sin_sg{k}")) for k in range(1, 5)]
    cos_sg = [None] + [c3(getattr(g, f"cos_sg{k}")) for k in range(1, 5)]
    dxc, dyc, dx, dy = c3(g.dxc), c3(g.dyc), c3(g.dx), c3(g.dy)
    rarea, rarea_c = c3(g.rarea), c3(g.rarea_c)
    shp = delp.shape
    # initialize_delpc_ptc (c_sw.py:372-376), full halo domain
    delpc = np.full(shp, np.nan)
    ptc = np.full(shp, np.nan)
    full = t.m - 1
    delpc[:full, :full, :nz] = 0.0
    ptc[:full, :full, :nz] = 0.0
    d2a2c_vect(t, g, uc, vc, u, v, ua, va, ut, vt)
    if nord > 0:
        # divergence_corner (c_sw.py:172-287): cell corners of the compute domain
        uf = (u - 0.25 * (sh(va, 0, -1) + va) * (sh(cos_sg[4], 0, -1) + cos_sg[2])) * dyc * 0.5 * (
            sh(sin_sg[4], 0, -1) + sin_sg[2]
        )
        vf = (v - 0.25 * (sh(ua, -1, 0) + ua) * (sh(cos_sg[3], -1, 0) + cos_sg[1])) * dxc * 0.5 * (
            sh(sin_sg[3], -1, 0) + sin_sg[1]
        )
        dd = (sh(vf, 0, -1) - vf + sh(uf, -1, 0) - uf) * rarea_c
        m_ew = at(t, i=s) | at(t, i=e + 1)
        vf0 = v * dxc * 0.5 * (sh(sin_sg[3], -1, 0) + sin_sg[1])
        vf1 = sh(v, 0, -1) * sh(dxc, 0, -1) * 0.5 * (sh(sin_sg[3], -1, -1) + sh(sin_sg[1], 0, -1))
        uf1 = (
            (sh(u, -1, 0) - 0.25 * (sh(va, -1, -1) + sh(va, -1, 0)) * (sh(cos_sg[4], -1, -1) + sh(cos_sg[2], -1, 0)))
            * sh(dyc, -1, 0)
            * 0.5
            * (sh(sin_sg[4], -1, -1) + sh(sin_sg[2], -1, 0))
        )
        dd = np.where(m_ew, (vf1 - vf0 + uf1 - uf) * rarea_c, dd)
        m_ns = at(t, j=js) | at(t, j=je + 1)
        uf0 = u * dyc * 0.5 * (sh(sin_sg[4], 0, -1) + sin_sg[2])
        uf1b = sh(u, -1, 0) * sh(dyc, -1, 0) * 0.5 * (sh(sin_sg[4], -1, -1) + sh(sin_sg[2], -1, 0))
        vf1b = (
            (sh(v, 0, -1) - 0.25 * (sh(ua, -1, -1) + sh(ua, 0, -1)) * (sh(cos_sg[3], -1, -1) + sh(cos_sg[1], 0, -1)))
            * sh(dxc, 0, -1)
            * 0.5
            * (sh(sin_sg[3], -1, -1) + sh(sin_sg[1], 0, -1))
        )
        dd = np.where(m_ns, (vf1b - vf + uf1b - uf0) * rarea_c, dd)
        m_sc = region(t, s, s + 1, js, js + 1) | region(t, e + 1, e + 2, js, js + 1)
        dd = np.where(m_sc, (-vf0 + uf1b - uf0) * rarea_c, dd)
        m_nc = region(t, e + 1, e + 2, je + 1, je + 2) | region(t, s, s + 1, je + 1, je + 2)
        dd = np.where(m_nc, (vf1 + uf1b - uf0) * rarea_c, dd)
        put(divgd, dd, s, e + 2, js, je + 2, 0, nz)
    # geoadjust_ut / vt (c_sw.py:20-43)
    utn = np.where(ut > 0, dt2 * ut * dy * sh(sin_sg[3], -1, 0), dt2 * ut * dy * sin_sg[1])
    put(ut, utn, s - 1, e + 3, js - 1, je + 2, 0, nz)
    vtn = np.where(vt > 0, dt2 * vt * dx * sh(sin_sg[4], 0, -1), dt2 * vt * dx * sin_sg[2])
    put(vt, vtn, s - 1, e + 2, js - 1, je + 3, 0, nz)
    # fill_corners_x on delp, pt, w (c_sw.py:51-64), in place
    for q in (delp, pt, w):
        put(q, corners.fill_corners_2cells_x(t, q), 0, full, 0, full, 0, nz)
    # compute_nonhydro_fluxes_x (c_sw.py:67-82)
    pos = ut > 0.0
    fx1 = ut * np.where(pos, sh(delp, -1, 0), delp)
    fx = fx1 * np.where(pos, sh(pt, -1, 0), pt)
    fx2 = fx1 * np.where(pos, sh(w, -1, 0), w)
    bx = (s - 1, e + 3, js - 1, je + 2)
    tfx = np.full(shp, np.nan)
    tfx1 = np.full(shp, np.nan)
    tfx2 = np.full(shp, np.nan)
    put(tfx1, fx1, *bx, 0, nz)
    put(tfx, fx, *bx, 0, nz)
    put(tfx2, fx2, *bx, 0, nz)
    # fill_corners_y on delp, pt, w
    for q in (delp, pt, w):
        put(q, corners.fill_corners_2cells_y(t, q), 0, full, 0, full, 0, nz)
    # transportdelp_update_vorticity_and_kineticenergy (c_sw.py:85-169)
    posy = vt > 0.0
    fy1 = vt * np.where(posy, sh(delp, 0, -1), delp)
    fy = fy1 * np.where(posy, sh(pt, 0, -1), pt)
    fy2 = fy1 * np.where(posy, sh(w, 0, -1), w)
    bc = (s - 1, e + 2, js - 1, je + 2)
    dpc = delp + (tfx1 - sh(tfx1, 1, 0) + fy1 - sh(fy1, 0, 1)) * rarea
    put(delpc, dpc, *bc, 0, nz)
    ptcv = (pt * delp + (tfx - sh(tfx, 1, 0) + fy - sh(fy, 0, 1)) * rarea) / delpc
    put(ptc, ptcv, *bc, 0, nz)
    wcv = (w * delp + (tfx2 - sh(tfx2, 1, 0) + fy2 - sh(fy2, 0, 1)) * rarea) / delpc
    put(omga, wcv, *bc, 0, nz)
    ke = np.where(ua > 0.0, uc, sh(uc, 1, 0))
    vort = np.where(va > 0.0, vc, sh(vc, 0, 1))
    m = at(t, j=js - 1) | at(t, j=je)
    vort = np.where(m & (va <= 0.0), vort * sin_sg[4] + sh(u, 0, 1) * cos_sg[4], vort)
    m = at(t, j=js) | at(t, j=je + 1)
    vort = np.where(m & (va > 0.0), vort * sin_sg[2] + u * cos_sg[2], vort)
    m = at(t, i=e) | at(t, i=s - 1)
    ke = np.where(m & (ua <= 0.0), ke * sin_sg[3] + sh(v, 1, 0) * cos_sg[3], ke)
    m = at(t, i=e + 1) | at(t, i=s)
    ke = np.where(m & (ua > 0.0), ke * sin_sg[1] + v * cos_sg[1], ke)
    ke = 0.5 * dt2 * (ua * ke + va * vort)
    tke = np.full(shp, np.nan)
    tvort = np.full(shp, np.nan)
    put(tke, ke, *bc, 0, nz)
    put(tvort, vort, *bc, 0, nz)
    # circulation_cgrid (c_sw.py:292-322)
    fxc = dxc * uc
    fyc = dyc * vc
    fx1c = sh(dxc, 0, -1) * sh(uc, 0, -1)
    fy1c = sh(dyc, -1, 0) * sh(vc, -1, 0)
    vc_ = fx1c - fxc - fy1c + fyc
    m = region(t, s, s + 1, js, js + 1) | region(t, s, s + 1, je + 1, je + 2)
    vc_ = np.where(m, fx1c - fxc + fyc, vc_)
    m = region(t, e + 1, e + 2, js, js + 1) | region(t, e + 1, e + 2, je + 1, je + 2)
    vc_ = np.where(m, fx1c - fxc - fy1c, vc_)
    put(tvort, vc_, s, e + 2, js, je + 2, 0, nz)
    # absolute_vorticity (c_sw.py:46-48)
    put(tvort, c3(fC) + rarea_c * tvort, s, e + 2, js, je + 2, 0, nz)
    # update_y_velocity (c_sw.py:349-369): vc on (X, Y_INTERFACE)
    tmp_flux = dt2 * (u - vc * c3(g.cosa_v)) / c3(g.sina_v)
    m = at(t, j=js) | at(t, j=je + 1)
    tmp_flux = np.where(m, dt2 * u, tmp_flux)
    flux = np.where(tmp_flux > 0.0, tvort, sh(tvort, 1, 0))
    put(vc, vc - tmp_flux * flux + c3(g.rdyc) * (sh(tke, 0, -1) - tke), s, e + 1, js, je + 2, 0, nz)
    # update_x_velocity (c_sw.py:325-346): uc on (X_INTERFACE, Y)
    tmp_flux = dt2 * (v - uc * c3(g.cosa_u)) / c3(g.sina_u)
    m = at(t, i=s) | at(t, i=e + 1)
    tmp_flux = np.where(m, dt2 * v, tmp_flux)
    flux = np.where(tmp_flux > 0.0, tvort, sh(tvort, 0, 1))
    put(uc, uc + tmp_flux * flux + c3(g.rdxc) * (sh(tke, -1, 0) - tke), s, e + 2, js, je + 1, 0, nz)
    return delpc, ptc
