"""Flux preparation (reference ``fv3core/stencils/fxadv.py``,
``FiniteVolumeFluxPrep.__call__`` 488-585): contravariant C-grid winds,
Courant numbers and area fluxes, with the 2x2 corner solves.

``uc_contra``/``vc_contra`` are storages the reference keeps between calls;
rows/columns it does not recompute keep their previous contents, so the
caller passes the same arrays every call.
"""
import numpy as np

from ._util import Tile, at, c3, put, region, sh


def _contra(v1, v2, cosa, rsin2):
    return (v1 - v2 * cosa) * rsin2


def fxadv(t: Tile, g, uc, vc, crx, cry, xfx, yfx, uc_contra, vc_contra, dt):
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    nz = t.nz
    full = t.m - 1
    cosa_u, cosa_v = c3(g.cosa_u), c3(g.cosa_v)
    rsin_u, rsin_v = c3(g.rsin_u), c3(g.rsin_v)
    sin_sg1, sin_sg2, sin_sg3, sin_sg4 = (c3(getattr(g, f"sin_sg{k}")) for k in range(1, 5))
    fb = (0, full, 0, full, 0, nz)  # full halo domain
    # main_uc_contra (fxadv.py:11-39)
    utmp = uc_contra.copy()
    vv = 0.25 * (sh(vc, -1, 0) + vc + sh(vc, -1, 1) + sh(vc, 0, 1))
    new = np.where(region(t, s - 1, e + 3, None, None), _contra(uc, vv, cosa_u, rsin_u), uc_contra)
    m = region(t, None, None, js - 1, js + 1) | region(t, None, None, je, je + 2)
    new = np.where(m, utmp, new)
    put(uc_contra, new, *fb)
    # uc_contra_y_edge (fxadv.py:61-71)
    m = at(t, i=s) | at(t, i=e + 1)
    new = np.where(m, np.where(uc > 0, uc / sh(sin_sg3, -1, 0), uc / sin_sg1), uc_contra)
    put(uc_contra, new, *fb)
    # main_vc_contra (fxadv.py:42-58)
    vtmp = vc_contra.copy()
    uu = 0.25 * (sh(uc, 0, -1) + sh(uc, 1, -1) + uc + sh(uc, 1, 0))
    new = np.where(region(t, None, None, js - 1, je + 3), _contra(vc, uu, cosa_v, rsin_v), vc_contra)
    m = at(t, j=js) | at(t, j=je + 1)
    new = np.where(m, vtmp, new)
    put(vc_contra, new, *fb)
    # vc_contra_y_edge (fxadv.py:97-137)
    vtmp = vc_contra.copy()
    m = region(t, s - 1, s + 1, js, je + 2) | region(t, e, e + 2, js, je + 2)
    u_c = 0.25 * (sh(uc_contra, 0, -1) + sh(uc_contra, 1, -1) + uc_contra + sh(uc_contra, 1, 0))
    new = np.where(m, _contra(vc, u_c, cosa_v, 1.0), vc_contra)
    m = (
        region(t, s - 1, s + 1, js, js + 2)
        | region(t, e, e + 2, js, js + 2)
        | region(t, s - 1, s + 1, je, je + 2)
        | region(t, e, e + 2, je, je + 2)
    )
    new = np.where(m, vtmp, new)
    put(vc_contra, new, *fb)
    # vc_contra_x_edge (fxadv.py:140-150)
    m = at(t, j=js) | at(t, j=je + 1)
    new = np.where(m, np.where(vc > 0, vc / sh(sin_sg4, 0, -1), vc / sin_sg2), vc_contra)
    put(vc_contra, new, *fb)
    # uc_contra_x_edge (fxadv.py:74-94)
    utmp = uc_contra.copy()
    m = region(t, s, e + 2, js - 1, js + 1) | region(t, s, e + 2, je, je + 2)
    v_c = 0.25 * (sh(vc_contra, -1, 0) + vc_contra + sh(vc_contra, -1, 1) + sh(vc_contra, 0, 1))
    new = np.where(m, _contra(uc, v_c, cosa_u, 1.0), uc_contra)
    m = (
        region(t, s, s + 2, js - 1, js + 1)
        | region(t, s, s + 2, je, je + 2)
        | region(t, e, e + 2, js - 1, js + 1)
        | region(t, e, e + 2, je, je + 2)
    )
    new = np.where(m, utmp, new)
    put(uc_contra, new, *fb)
    # uc_contra_corners (fxadv.py:156-260); domain starts one point in
    cb = (1, full, 1, full, 0, nz)
    uci, vci, uco = uc, vc_contra, uc_contra  # uc_contra is aliased as its own copy
    damp = 1.0 / (1.0 - 0.0625 * cosa_u * sh(cosa_v, -1, 0))
    val = (
        uci - 0.25 * cosa_u * (sh(vci, -1, 1) + sh(vci, 0, 1) + vci + sh(vc, -1, 0)
                               - 0.25 * sh(cosa_v, -1, 0) * (sh(uco, -1, 0) + sh(uco, -1, -1) + sh(uco, 0, -1)))
    ) * damp
    m = region(t, s + 1, s + 2, js - 1, js) | region(t, s + 1, s + 2, je, je + 1)
    put(uc_contra, np.where(m, val, uc_contra), *cb)
    damp = 1.0 / (1.0 - 0.0625 * cosa_u * sh(cosa_v, -1, 1))
    val = (
        uci - 0.25 * cosa_u * (sh(vci, -1, 0) + vci + sh(vci, 0, 1) + sh(vc, -1, 1)
                               - 0.25 * sh(cosa_v, -1, 1) * (sh(uco, -1, 0) + sh(uco, -1, 1) + sh(uco, 0, 1)))
    ) * damp
    m = region(t, s + 1, s + 2, js, js + 1) | region(t, s + 1, s + 2, je + 1, je + 2)
    put(uc_contra, np.where(m, val, uc_contra), *cb)
    damp = 1.0 / (1.0 - 0.0625 * cosa_u * cosa_v)
    val = (
        uci - 0.25 * cosa_u * (sh(vci, 0, 1) + sh(vci, -1, 1) + sh(vci, -1, 0) + vc
                               - 0.25 * cosa_v * (sh(uco, 1, 0) + sh(uco, 1, -1) + sh(uco, 0, -1)))
    ) * damp
    m = region(t, e, e + 1, js - 1, js) | region(t, e, e + 1, je, je + 1)
    put(uc_contra, np.where(m, val, uc_contra), *cb)
    damp = 1.0 / (1.0 - 0.0625 * cosa_u * sh(cosa_v, 0, 1))
    val = (
        uci - 0.25 * cosa_u * (vci + sh(vci, -1, 0) + sh(vci, -1, 1) + sh(vc, 0, 1)
                               - 0.25 * sh(cosa_v, 0, 1) * (sh(uco, 1, 0) + sh(uco, 1, 1) + sh(uco, 0, 1)))
    ) * damp
    m = region(t, e, e + 1, js, js + 1) | region(t, e, e + 1, je + 1, je + 2)
    put(uc_contra, np.where(m, val, uc_contra), *cb)
    # vc_contra_corners (fxadv.py:263-383); vc_contra aliased as its copy
    ut = uc_contra
    vco = vc_contra
    damp = 1.0 / (1.0 - 0.0625 * sh(cosa_u, 0, -1) * cosa_v)
    val = (
        vc - 0.25 * cosa_v * (sh(ut, 1, -1) + sh(ut, 1, 0) + ut + sh(uc, 0, -1)
                              - 0.25 * sh(cosa_u, 0, -1) * (sh(vco, 0, -1) + sh(vco, -1, -1) + sh(vco, -1, 0)))
    ) * damp
    m = region(t, s - 1, s, js + 1, js + 2) | region(t, e, e + 1, js + 1, js + 2)
    put(vc_contra, np.where(m, val, vc_contra), *cb)
    damp = 1.0 / (1.0 - 0.0625 * sh(cosa_u, 1, -1) * cosa_v)
    val = (
        vc - 0.25 * cosa_v * (sh(ut, 0, -1) + ut + sh(ut, 1, 0) + sh(uc, 1, -1)
                              - 0.25 * sh(cosa_u, 1, -1) * (sh(vco, 0, -1) + sh(vco, 1, -1) + sh(vco, 1, 0)))
    ) * damp
    m = region(t, s, s + 1, js + 1, js + 2) | region(t, e + 1, e + 2, js + 1, js + 2)
    put(vc_contra, np.where(m, val, vc_contra), *cb)
    damp = 1.0 / (1.0 - 0.0625 * sh(cosa_u, 1, 0) * cosa_v)
    val = (
        vc - 0.25 * cosa_v * (ut + sh(ut, 0, -1) + sh(ut, 1, -1) + sh(uc, 1, 0)
                              - 0.25 * sh(cosa_u, 1, 0) * (sh(vco, 0, 1) + sh(vco, 1, 1) + sh(vco, 1, 0)))
    ) * damp
    m = region(t, e + 1, e + 2, je, je + 1) | region(t, s, s + 1, je, je + 1)
    put(vc_contra, np.where(m, val, vc_contra), *cb)
    damp = 1.0 / (1.0 - 0.0625 * cosa_u * cosa_v)
    val = (
        vc - 0.25 * cosa_v * (sh(ut, 1, 0) + sh(ut, 1, -1) + sh(ut, 0, -1) + uc
                              - 0.25 * cosa_u * (sh(vco, 0, 1) + sh(vco, -1, 1) + sh(vco, -1, 0)))
    ) * damp
    m = region(t, e, e + 1, je, je + 1) | region(t, s - 1, s, je, je + 1)
    put(vc_contra, np.where(m, val, vc_contra), *cb)
    # fxadv_fluxes_stencil (fxadv.py:386-421)
    prod = dt * uc_contra
    pos = prod > 0
    m = region(t, s, e + 2, None, None)
    put(crx, np.where(pos, prod * sh(c3(g.rdxa), -1, 0), prod * c3(g.rdxa)), *fb, mask=m)
    put(xfx, np.where(pos, c3(g.dy) * prod * sh(sin_sg3, -1, 0), c3(g.dy) * prod * sin_sg1), *fb, mask=m)
    prod = dt * vc_contra
    pos = prod > 0
    m = region(t, None, None, js, je + 2)
    put(cry, np.where(pos, prod * sh(c3(g.rdya), 0, -1), prod * c3(g.rdya)), *fb, mask=m)
    put(yfx, np.where(pos, c3(g.dx) * prod * sh(sin_sg4, 0, -1), c3(g.dx) * prod * sin_sg2), *fb, mask=m)
