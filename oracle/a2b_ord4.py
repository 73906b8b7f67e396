"""Fourth-order A-grid to B-grid interpolation (reference
``fv3core/stencils/a2b_ord4.py``, ``AGrid2BGridFourthOrder.__call__``
606-676), applied on levels [k0, k1).

``tmp_qout_edges`` is a storage the reference keeps between calls (NaN
until first written).
"""
import numpy as np

from ._util import Tile, at, c3, put, sh

# a2b_ord4.py:24-35
C1, C2 = 2.0 / 3.0, -1.0 / 6.0
B1, B2 = 7.0 / 12.0, -1.0 / 12.0
A1, A2 = 9.0 / 16.0, -1.0 / 16.0


def _s(a, d, axis):
    return sh(a, d, 0) if axis == 0 else sh(a, 0, d)


def great_circle_dist(p1a, p1b, p2a, p2b):
    """a2b_ord4.py:38-41."""
    tb = np.sin((p1b - p2b) / 2.0) ** 2.0
    ta = np.sin((p1a - p2a) / 2.0) ** 2.0
    return np.arcsin(np.sqrt(tb + np.cos(p1b) * np.cos(p2b) * ta)) * 2.0


def extrap_corner(p0a, p0b, p1a, p1b, p2a, p2b, qa, qb):
    """a2b_ord4.py:45-57."""
    x1 = great_circle_dist(p1a, p1b, p0a, p0b)
    x2 = great_circle_dist(p2a, p2b, p0a, p0b)
    return qa + x1 / (x2 - x1) * (qa - qb)


def _corner_value(g, qin, i, j, offsets):
    """(ec1 + ec2 + ec3) / 3 at B-grid point (i, j); ``offsets`` lists the
    (near, far) A-grid offsets of the three extrapolations."""
    b1, b2 = g.bgrid1[i, j], g.bgrid2[i, j]
    ecs = []
    for (di1, dj1), (di2, dj2) in offsets:
        ecs.append(
            extrap_corner(
                b1, b2,
                g.agrid1[i + di1, j + dj1], g.agrid2[i + di1, j + dj1],
                g.agrid1[i + di2, j + dj2], g.agrid2[i + di2, j + dj2],
                qin[i + di1, j + dj1], qin[i + di2, j + dj2],
            )
        )
    return (ecs[0] + ecs[1] + ecs[2]) * (1.0 / 3.0)


_SW = [((0, 0), (1, 1)), ((-1, 0), (-2, 1)), ((0, -1), (1, -2))]  # a2b_ord4.py:60-103
_NW = [((-1, 0), (-2, 1)), ((-1, -1), (-2, -2)), ((0, 0), (1, 1))]  # 106-147
_NE = [((-1, -1), (-2, -2)), ((0, -1), (1, -2)), ((-1, 0), (-2, 1))]  # 150-191
_SE = [((0, -1), (1, -2)), ((-1, -1), (-2, -2)), ((0, 0), (1, 1))]  # 194-235


def _qx_edge_1(qin, dxa, axis):
    """qx_edge_west (a2b_ord4.py:340-350) / qy_edge_south."""
    g_in = _s(dxa, 1, axis) / dxa
    g_ou = _s(dxa, -2, axis) / _s(dxa, -1, axis)
    return 0.5 * (
        ((2.0 + g_in) * qin - _s(qin, 1, axis)) / (1.0 + g_in)
        + ((2.0 + g_ou) * _s(qin, -1, axis) - _s(qin, -2, axis)) / (1.0 + g_ou)
    )


def _qx_edge_2(qin, dxa, axis):
    """qx_edge_west2 (a2b_ord4.py:354-368) / qy_edge_south2."""
    g_in = dxa / _s(dxa, -1, axis)
    g_ou = _s(dxa, -3, axis) / _s(dxa, -2, axis)
    left = 0.5 * (
        ((2.0 + g_in) * _s(qin, -1, axis) - qin) / (1.0 + g_in)
        + ((2.0 + g_ou) * _s(qin, -2, axis) - _s(qin, -3, axis)) / (1.0 + g_ou)
    )
    right = B2 * (_s(qin, -1, axis) + _s(qin, 2, axis)) + B1 * (qin + _s(qin, 1, axis))
    return (3.0 * (g_in * _s(qin, -1, axis) + qin) - (g_in * left + right)) / (2.0 + 2.0 * g_in)


def _qx_edge_3(qin, dxa, axis):
    """qx_edge_east (a2b_ord4.py:372-378) / qy_edge_north."""
    g_in = _s(dxa, -2, axis) / _s(dxa, -1, axis)
    g_ou = _s(dxa, 1, axis) / dxa
    return 0.5 * (
        ((2.0 + g_in) * _s(qin, -1, axis) - _s(qin, -2, axis)) / (1.0 + g_in)
        + ((2.0 + g_ou) * qin - _s(qin, 1, axis)) / (1.0 + g_ou)
    )


def _qx_edge_4(qin, dxa, axis):
    """qx_edge_east2 (a2b_ord4.py:382-395) / qy_edge_north2."""
    g_in = _s(dxa, -1, axis) / dxa
    g_ou = _s(dxa, 2, axis) / _s(dxa, 1, axis)
    right = 0.5 * (
        ((2.0 + g_in) * qin - _s(qin, -1, axis)) / (1.0 + g_in)
        + ((2.0 + g_ou) * _s(qin, 1, axis) - _s(qin, 2, axis)) / (1.0 + g_ou)
    )
    left = B2 * (_s(qin, -3, axis) + qin) + B1 * (_s(qin, -2, axis) + _s(qin, -1, axis))
    return (3.0 * (_s(qin, -1, axis) + g_in * qin) - (g_in * right + left)) / (2.0 + 2.0 * g_in)


def ppm_volume_mean(t: Tile, qin, dxa, axis):
    """ppm_volume_mean_x / _y (a2b_ord4.py:248-283), full-tile array."""
    dxa = c3(dxa)
    q = B2 * (_s(qin, -2, axis) + _s(qin, 1, axis)) + B1 * (_s(qin, -1, axis) + qin)
    s = t.isc if axis == 0 else t.jsc
    e = t.iec if axis == 0 else t.jec

    def line(idx):
        return at(t, i=idx) if axis == 0 else at(t, j=idx)

    q = np.where(line(s), _qx_edge_1(qin, dxa, axis), q)
    q = np.where(line(s + 1), _qx_edge_2(qin, dxa, axis), q)
    q = np.where(line(e + 1), _qx_edge_3(qin, dxa, axis), q)
    q = np.where(line(e), _qx_edge_4(qin, dxa, axis), q)
    return q


class A2BScratch:
    def __init__(self, shape):
        self.qx = np.full(shape, np.nan)
        self.qy = np.full(shape, np.nan)
        self.tmp_qout_edges = np.full(shape, np.nan)


def a2b_ord4(t: Tile, g, qin, qout, k0, k1, scr: A2BScratch, replace=False):
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    dxa, dya = c3(g.dxa), c3(g.dya)
    T = scr.tmp_qout_edges
    ks = slice(k0, k1)
    # corner values (a2b_ord4.py:616-654): the reference's stencil names
    # _nw/_se are applied at the (ie+1, js) / (is, je+1) corners
    for (i, j), offs in (((s, js), _SW), ((e + 1, js), _NW), ((e + 1, je + 1), _NE), ((s, je + 1), _SE)):
        v = _corner_value(g, qin[:, :, ks], i, j, offs)
        qout[i, j, ks] = v
        T[i, j, ks] = v
    # edges (a2b_ord4.py:313-336, 678-695)
    for ii, ew in ((s, g.edge_w), (e + 1, g.edge_e)):
        for j in range(js + 1, je + 1):
            def q2(jj):
                return (qin[ii - 1, jj, ks] * g.dxa[ii, jj] + qin[ii, jj, ks] * g.dxa[ii - 1, jj]) / (
                    g.dxa[ii - 1, jj] + g.dxa[ii, jj]
                )

            w = ew[j - t.h]
            v = w * q2(j - 1) + (1.0 - w) * q2(j)
            qout[ii, j, ks] = v
            T[ii, j, ks] = v
    for jj, es in ((js, g.edge_s), (je + 1, g.edge_n)):
        for i in range(s + 1, e + 1):
            def q1(ii):
                return (qin[ii, jj - 1, ks] * g.dya[ii, jj] + qin[ii, jj, ks] * g.dya[ii, jj - 1]) / (
                    g.dya[ii, jj - 1] + g.dya[ii, jj]
                )

            w = es[i - t.h]
            v = w * q1(i - 1) + (1.0 - w) * q1(i)
            qout[i, jj, ks] = v
            T[i, jj, ks] = v
    # ppm volume means: qx on [is, ie+1] x [js-2, je+2], qy on [is-2, ie+2] x [js, je+1]
    scr.qx[s : e + 2, js - 2 : je + 3, ks] = ppm_volume_mean(t, qin, dxa, 0)[s : e + 2, js - 2 : je + 3, ks]
    scr.qy[s - 2 : e + 3, js : je + 2, ks] = ppm_volume_mean(t, qin, dya, 1)[s - 2 : e + 3, js : je + 2, ks]
    qx, qy = scr.qx, scr.qy
    # a2b_interpolation (a2b_ord4.py:286-310) on interior corners
    qxx = A2 * (sh(qx, 0, -2) + sh(qx, 0, 1)) + A1 * (sh(qx, 0, -1) + qx)
    qyy = A2 * (sh(qy, -2, 0) + sh(qy, 1, 0)) + A1 * (sh(qy, -1, 0) + qy)
    up = A2 * (sh(qx, 0, -1) + sh(qx, 0, 2)) + A1 * (qx + sh(qx, 0, 1))
    qxx = np.where(at(t, j=js + 1), C1 * (sh(qx, 0, -1) + qx) + C2 * (sh(T, 0, -1) + up), qxx)
    lo = A2 * (sh(qx, 0, -3) + qx) + A1 * (sh(qx, 0, -2) + sh(qx, 0, -1))
    qxx = np.where(at(t, j=je), C1 * (sh(qx, 0, -1) + qx) + C2 * (sh(T, 0, 1) + lo), qxx)
    right = A2 * (sh(qy, -1, 0) + sh(qy, 2, 0)) + A1 * (qy + sh(qy, 1, 0))
    qyy = np.where(at(t, i=s + 1), C1 * (sh(qy, -1, 0) + qy) + C2 * (sh(T, -1, 0) + right), qyy)
    left = A2 * (sh(qy, -3, 0) + qy) + A1 * (sh(qy, -2, 0) + sh(qy, -1, 0))
    qyy = np.where(at(t, i=e), C1 * (sh(qy, -1, 0) + qy) + C2 * (sh(T, 1, 0) + left), qyy)
    val = 0.5 * (qxx + qyy)
    qout[s + 1 : e + 1, js + 1 : je + 1, ks] = val[s + 1 : e + 1, js + 1 : je + 1, ks]
    if replace:
        qin[s : e + 2, js : je + 2, ks] = qout[s : e + 2, js : je + 2, ks]
