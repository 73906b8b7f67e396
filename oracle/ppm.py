"""Piecewise-parabolic fluxes (reference ``fv3core/stencils/xppm.py``,
``yppm.py``, ``ppm.py``) and the wind self-advection of the kinetic-energy
term (``xtp_u.py``, ``ytp_v.py``).

Both branches are restated: the monotonic ``mord < 8`` one (hord 5/6, the
acoustic substep) and the ord-8 limiter of tracer transport (hord_tr = 8,
xppm.py:85-266).  Functions return full-tile arrays; callers store the
reference's domain.
The y-direction versions are the x versions with the axes exchanged, as in
the reference (yppm.py is generated from xppm.py).
"""
import numpy as np

from ._util import Tile, at, c3, sh

# ppm.py:8-20
PC1, PC2, PC3 = -2.0 / 14.0, 11.0 / 14.0, 5.0 / 14.0
P1, P2 = 7.0 / 12.0, -1.0 / 12.0
S11, S14, S15 = 11.0 / 14.0, 4.0 / 7.0, 3.0 / 14.0


def _s(a, d, axis):
    return sh(a, d, 0) if axis == 0 else sh(a, 0, d)


def compute_al(t: Tile, q, dxa, axis, iord=6):
    """xppm.py:148-181 (axis 0) / yppm.py compute_al (axis 1)."""
    if iord < 0:
        raise NotImplementedError("negative iord")
    dxa = c3(dxa)
    al = P1 * (_s(q, -1, axis) + q) + P2 * (_s(q, -2, axis) + _s(q, 1, axis))
    s = t.isc if axis == 0 else t.jsc
    e = t.iec if axis == 0 else t.jec

    def line(idx):
        return at(t, i=idx) if axis == 0 else at(t, j=idx)

    m = line(s - 1) | line(e)
    al = np.where(m, PC1 * _s(q, -2, axis) + PC2 * _s(q, -1, axis) + PC3 * q, al)
    m = line(s) | line(e + 1)
    edge = 0.5 * (
        ((2.0 * _s(dxa, -1, axis) + _s(dxa, -2, axis)) * _s(q, -1, axis) - _s(dxa, -1, axis) * _s(q, -2, axis))
        / (_s(dxa, -2, axis) + _s(dxa, -1, axis))
        + ((2.0 * dxa + _s(dxa, 1, axis)) * q - dxa * _s(q, 1, axis)) / (dxa + _s(dxa, 1, axis))
    )
    al = np.where(m, edge, al)
    m = line(s + 1) | line(e + 2)
    al = np.where(m, PC3 * _s(q, -1, axis) + PC2 * q + PC1 * _s(q, 1, axis), al)
    return al


def fx1_fn(courant, br, b0, bl, axis):
    """xppm.py:32-44."""
    return np.where(
        courant > 0.0,
        (1.0 - courant) * (_s(br, -1, axis) - courant * _s(b0, -1, axis)),
        (1.0 + courant) * (bl + courant * b0),
    )


def advection_mask(bl, b0, br, axis, mord=6):
    """xppm.py:48-61."""
    if mord == 5:
        smt5 = bl * br < 0
    else:
        smt5 = (3.0 * np.abs(b0)) < np.abs(bl - br)
    prev = _s(smt5.astype(np.float64), -1, axis)
    return np.where((prev != 0) | smt5, 1.0, 0.0)


def apply_flux(courant, q, fx1, mask, axis):
    """xppm.py:19-28."""
    return np.where(courant > 0.0, _s(q, -1, axis) + fx1 * mask, q + fx1 * mask)


def sign(a, b):
    """basic_operations.sign (basic_operations.py:34-40): |a| with the sign
    of b, negative unless b > 0."""
    return np.where(b > 0, np.abs(a), -np.abs(a))


def dm_iord8plus(q, axis):
    """xppm.py:85-90."""
    xt = 0.25 * (_s(q, 1, axis) - _s(q, -1, axis))
    dqr = np.maximum(np.maximum(q, _s(q, -1, axis)), _s(q, 1, axis)) - q
    dql = q - np.minimum(np.minimum(q, _s(q, -1, axis)), _s(q, 1, axis))
    return sign(np.minimum(np.minimum(np.abs(xt), dqr), dql), xt)


def _dm_shifted(q, axis, d):
    """The dm_left / dm_right temporaries of bl_br_edges (xppm.py:191-236):
    dm_iord8plus of the neighbour at offset d, written out."""
    qm, q0, qp = _s(q, d - 1, axis), _s(q, d, axis), _s(q, d + 1, axis)
    xt = 0.25 * (qp - qm)
    dqr = np.maximum(np.maximum(q0, qm), qp) - q0
    dql = q0 - np.minimum(np.minimum(q0, qm), qp)
    return sign(np.minimum(np.minimum(np.abs(xt), dqr), dql), xt)


def _xt_dxa_edge_0(q, dxa, axis):
    """xt_dxa_edge_0 with xt_minmax (xppm.py:109-131)."""
    xt = 0.5 * (
        ((2.0 * dxa + _s(dxa, -1, axis)) * q - dxa * _s(q, -1, axis)) / (_s(dxa, -1, axis) + dxa)
        + ((2.0 * _s(dxa, 1, axis) + _s(dxa, 2, axis)) * _s(q, 1, axis) - _s(dxa, 1, axis) * _s(q, 2, axis))
        / (_s(dxa, 1, axis) + _s(dxa, 2, axis))
    )
    minq = np.minimum(np.minimum(np.minimum(_s(q, -1, axis), q), _s(q, 1, axis)), _s(q, 2, axis))
    maxq = np.maximum(np.maximum(np.maximum(_s(q, -1, axis), q), _s(q, 1, axis)), _s(q, 2, axis))
    return np.minimum(np.maximum(xt, minq), maxq)


def _xt_dxa_edge_1(q, dxa, axis):
    """xt_dxa_edge_1 with xt_minmax (xppm.py:118-145)."""
    xt = 0.5 * (
        ((2.0 * _s(dxa, -1, axis) + _s(dxa, -2, axis)) * _s(q, -1, axis) - _s(dxa, -1, axis) * _s(q, -2, axis))
        / (_s(dxa, -2, axis) + _s(dxa, -1, axis))
        + ((2.0 * dxa + _s(dxa, 1, axis)) * q - dxa * _s(q, 1, axis)) / (dxa + _s(dxa, 1, axis))
    )
    minq = np.minimum(np.minimum(np.minimum(_s(q, -2, axis), _s(q, -1, axis)), q), _s(q, 1, axis))
    maxq = np.maximum(np.maximum(np.maximum(_s(q, -2, axis), _s(q, -1, axis)), q), _s(q, 1, axis))
    return np.minimum(np.maximum(xt, minq), maxq)


def pert_ppm_standard_constraint(bl, br):
    """pert_ppm_standard_constraint_fcn (ppm.py:22-36) on (al, ar) = (bl, br)."""
    da1 = bl - br
    da2 = da1 ** 2
    a6da = 3.0 * (bl + br) * da1
    neg = bl * br < 0.0
    br_new = np.where(neg & (a6da < -da2), -2.0 * bl, br)
    bl_new = np.where(neg & ~(a6da < -da2) & (a6da > da2), -2.0 * br, bl)
    return np.where(neg, bl_new, 0.0), np.where(neg, br_new, 0.0)


def compute_blbr_ord8plus(t: Tile, q, dxa, axis):
    """compute_blbr_ord8plus (xppm.py:250-266): the ord-8 edge
    perturbations bl, br of every cell, with the tile-edge rules of
    bl_br_edges (xppm.py:185-246) and the standard constraint near the
    edges."""
    dxa = c3(dxa)
    dm = dm_iord8plus(q, axis)
    al = 0.5 * (_s(q, -1, axis) + q) + 1.0 / 3.0 * (_s(dm, -1, axis) - dm)
    # blbr_iord8 (xppm.py:98-102)
    xt = 2.0 * dm
    bl = -1.0 * sign(np.minimum(np.abs(xt), np.abs(al - q)), xt)
    br = sign(np.minimum(np.abs(xt), np.abs(_s(al, 1, axis) - q)), xt)
    s = t.isc if axis == 0 else t.jsc
    e = t.iec if axis == 0 else t.jec

    def line(idx):
        return at(t, i=idx) if axis == 0 else at(t, j=idx)

    qm1, qp1 = _s(q, -1, axis), _s(q, 1, axis)
    al_ip1 = _s(al, 1, axis)
    # each region's (xt_bl, xt_br), xppm.py:191-241
    rules = [
        (s - 1, S14 * _dm_shifted(q, axis, -1) + S11 * (qm1 - q) + q, _xt_dxa_edge_0(q, dxa, axis)),
        (s, _xt_dxa_edge_1(q, dxa, axis), S15 * q + S11 * qp1 - S14 * _dm_shifted(q, axis, 1)),
        (s + 1, S15 * qm1 + S11 * q - S14 * dm, al_ip1),
        (e - 1, al, S15 * qp1 + S11 * q + S14 * dm),
        (e, S15 * q + S11 * qm1 + S14 * _dm_shifted(q, axis, -1), _xt_dxa_edge_0(q, dxa, axis)),
        (e + 1, _xt_dxa_edge_1(q, dxa, axis), S11 * (qp1 - q) - S14 * _dm_shifted(q, axis, 1) + q),
    ]
    edge = np.zeros(bl.shape, dtype=bool) | line(s - 1)
    for idx, xbl, xbr in rules:
        m = line(idx)
        edge = edge | m
        bl = np.where(m, xbl - q, bl)
        br = np.where(m, xbr - q, br)
    cbl, cbr = pert_ppm_standard_constraint(bl, br)
    return np.where(edge, cbl, bl), np.where(edge, cbr, br)


def ppm_flux(t: Tile, q, courant, dxa, axis, iord=6):
    """compute_x_flux / compute_y_flux (xppm.py:269-280): the mean value of q
    advected through each interface."""
    mord = abs(iord)
    if mord >= 8:
        if iord != 8:
            raise NotImplementedError("only iord = 8 of the ord-8 family is implemented (as the reference)")
        bl, br = compute_blbr_ord8plus(t, q, dxa, axis)
        b0 = bl + br
        fx1 = fx1_fn(courant, br, b0, bl, axis)
        return apply_flux(courant, q, fx1, 1.0, axis)
    al = compute_al(t, q, dxa, axis, iord)
    bl = al - q
    br = _s(al, 1, axis) - q
    b0 = bl + br
    mask = advection_mask(bl, b0, br, axis, mord)
    fx1 = fx1_fn(courant, br, b0, bl, axis)
    return apply_flux(courant, q, fx1, mask, axis)


def advect_along(t: Tile, u, ub_contra, rdx, dx, dxa, dt, axis, iord=6):
    """advect_u_along_x (xtp_u.py:53-91) for axis 0 and advect_v_along_y
    (ytp_v.py) for axis 1, with get_bl_br (xtp_u.py:9-49)."""
    if iord >= 8:
        raise NotImplementedError("ord-8 PPM is not on the acoustic path")
    al = compute_al(t, u, dx, axis, iord)
    bl = al - u
    br = _s(al, 1, axis) - u
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    from ._util import region

    if axis == 0:
        zc = (
            region(t, s - 1, s + 1, js, js + 1)
            | region(t, s - 1, s + 1, je + 1, je + 2)
            | region(t, e, e + 2, js, js + 1)
            | region(t, e, e + 2, je + 1, je + 2)
        )
    else:
        zc = (
            region(t, s, s + 1, js - 1, js + 1)
            | region(t, e + 1, e + 2, js - 1, js + 1)
            | region(t, s, s + 1, je, je + 2)
            | region(t, e + 1, e + 2, je, je + 2)
        )
    bl = np.where(zc, 0.0, bl)
    br = np.where(zc, 0.0, br)
    b0 = bl + br
    rdx = c3(rdx)
    cfl = np.where(ub_contra > 0, ub_contra * dt * _s(rdx, -1, axis), ub_contra * dt * rdx)
    fx0 = fx1_fn(cfl, br, b0, bl, axis)
    mask = advection_mask(bl, b0, br, axis, abs(iord))
    return apply_flux(ub_contra, u, fx0, mask, axis)
