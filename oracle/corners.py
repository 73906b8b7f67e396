"""Cube-corner fills (reference ``fv3core/utils/corners.py``).

Each function returns a new full array equal to ``q`` except in the corner
halo cells named by the reference function, which are copied (times a
multiplier) from ``q_corner``.  Indices are absolute storage indices of one
tile; reads always see the values before the fill, as in the reference
where the filled field is a fresh temporary.
"""
import numpy as np

from ._util import Tile, at, sh


def _apply(t, q, q_corner, rules):
    out = np.array(q, copy=True)
    for (i, j, di, dj, mult) in rules:
        if 0 <= i < t.m and 0 <= j < t.m:
            out[i, j] = mult * q_corner[i + di, j + dj]
    return out


def fill_corners_2cells_mult_x(t: Tile, q, q_corner, sw, se, nw, ne):
    """corners.py:128-184."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    rules = [
        (s - 1, js - 1, 0, 1, sw),
        (s - 2, js - 1, 1, 2, sw),
        (e + 1, js - 1, 0, 1, se),
        (e + 2, js - 1, -1, 2, se),
        (s - 1, je + 1, 0, -1, nw),
        (s - 2, je + 1, 1, -2, nw),
        (e + 1, je + 1, 0, -1, ne),
        (e + 2, je + 1, -1, -2, ne),
    ]
    return _apply(t, q, q_corner, rules)


def fill_corners_3cells_mult_x(t: Tile, q, q_corner, sw, se, nw, ne):
    """corners.py:187-219."""
    out = fill_corners_2cells_mult_x(t, q, q_corner, sw, se, nw, ne)
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    rules = [
        (s - 3, js - 1, 2, 3, sw),
        (e + 3, js - 1, -2, 3, se),
        (s - 3, je + 1, 2, -3, nw),
        (e + 3, je + 1, -2, -3, ne),
    ]
    return _apply(t, out, q_corner, rules)


def fill_corners_2cells_mult_y(t: Tile, q, q_corner, sw, se, nw, ne):
    """corners.py:222-268."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    rules = [
        (s - 1, js - 1, 1, 0, sw),
        (s - 1, js - 2, 2, 1, sw),
        (e + 1, js - 1, -1, 0, se),
        (e + 1, js - 2, -2, 1, se),
        (s - 1, je + 1, 1, 0, nw),
        (s - 1, je + 2, 2, -1, nw),
        (e + 1, je + 1, -1, 0, ne),
        (e + 1, je + 2, -2, -1, ne),
    ]
    return _apply(t, q, q_corner, rules)


def fill_corners_3cells_mult_y(t: Tile, q, q_corner, sw, se, nw, ne):
    """corners.py:271-303."""
    out = fill_corners_2cells_mult_y(t, q, q_corner, sw, se, nw, ne)
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    rules = [
        (s - 1, js - 3, 3, 2, sw),
        (e + 1, js - 3, -3, 2, se),
        (s - 1, je + 3, 3, -2, nw),
        (e + 1, je + 3, -3, -2, ne),
    ]
    return _apply(t, out, q_corner, rules)


def fill_corners_2cells_x(t, q):
    return fill_corners_2cells_mult_x(t, q, q, 1.0, 1.0, 1.0, 1.0)


def fill_corners_2cells_y(t, q):
    return fill_corners_2cells_mult_y(t, q, q, 1.0, 1.0, 1.0, 1.0)


# copy_corners (corners.py:306-535): (target offset from the corner, source offset)
def _copy_rules_x(t):
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    R = []
    # south-west / south-east blocks (j = js-3 .. js-1)
    R += [((s - 3, js - 3), (0, 5)), ((e + 3, js - 3), (0, 5))]
    R += [((s - 2, js - 3), (-1, 4)), ((e + 3, js - 2), (-1, 4))]
    R += [((s - 1, js - 3), (-2, 3)), ((e + 3, js - 1), (-2, 3))]
    R += [((s - 3, js - 2), (1, 4)), ((e + 2, js - 3), (1, 4))]
    R += [((s - 2, js - 2), (0, 3)), ((e + 2, js - 2), (0, 3))]
    R += [((s - 1, js - 2), (-1, 2)), ((e + 2, js - 1), (-1, 2))]
    R += [((s - 3, js - 1), (2, 3)), ((e + 1, js - 3), (2, 3))]
    R += [((s - 2, js - 1), (1, 2)), ((e + 1, js - 2), (1, 2))]
    R += [((s - 1, js - 1), (0, 1)), ((e + 1, js - 1), (0, 1))]
    # north blocks
    R += [((s - 3, je + 1), (2, -3)), ((e + 1, je + 3), (2, -3))]
    R += [((s - 2, je + 1), (1, -2)), ((e + 1, je + 2), (1, -2))]
    R += [((s - 1, je + 1), (0, -1)), ((e + 1, je + 1), (0, -1))]
    R += [((s - 3, je + 2), (1, -4)), ((e + 2, je + 3), (1, -4))]
    R += [((s - 2, je + 2), (0, -3)), ((e + 2, je + 2), (0, -3))]
    R += [((s - 1, je + 2), (-1, -2)), ((e + 2, je + 1), (-1, -2))]
    R += [((s - 3, je + 3), (0, -5)), ((e + 3, je + 3), (0, -5))]
    R += [((s - 2, je + 3), (-1, -4)), ((e + 3, je + 2), (-1, -4))]
    R += [((s - 1, je + 3), (-2, -3)), ((e + 3, je + 1), (-2, -3))]
    return R


def _copy_rules_y(t):
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    R = []
    R += [((s - 3, js - 3), (5, 0)), ((s - 3, je + 3), (5, 0))]
    R += [((s - 2, js - 3), (4, 1)), ((s - 3, je + 2), (4, 1))]
    R += [((s - 1, js - 3), (3, 2)), ((s - 3, je + 1), (3, 2))]
    R += [((s - 3, js - 2), (4, -1)), ((s - 2, je + 3), (4, -1))]
    R += [((s - 2, js - 2), (3, 0)), ((s - 2, je + 2), (3, 0))]
    R += [((s - 1, js - 2), (2, 1)), ((s - 2, je + 1), (2, 1))]
    R += [((s - 3, js - 1), (3, -2)), ((s - 1, je + 3), (3, -2))]
    R += [((s - 2, js - 1), (2, -1)), ((s - 1, je + 2), (2, -1))]
    R += [((s - 1, js - 1), (1, 0)), ((s - 1, je + 1), (1, 0))]
    R += [((e + 1, js - 3), (-3, 2)), ((e + 3, je + 1), (-3, 2))]
    R += [((e + 2, js - 3), (-4, 1)), ((e + 3, je + 2), (-4, 1))]
    R += [((e + 3, js - 3), (-5, 0)), ((e + 3, je + 3), (-5, 0))]
    R += [((e + 1, js - 2), (-2, 1)), ((e + 2, je + 1), (-2, 1))]
    R += [((e + 2, js - 2), (-3, 0)), ((e + 2, je + 2), (-3, 0))]
    R += [((e + 3, js - 2), (-4, -1)), ((e + 2, je + 3), (-4, -1))]
    R += [((e + 1, js - 1), (-1, 0)), ((e + 1, je + 1), (-1, 0))]
    R += [((e + 2, js - 1), (-2, -1)), ((e + 1, je + 2), (-2, -1))]
    R += [((e + 3, js - 1), (-3, -2)), ((e + 1, je + 3), (-3, -2))]
    return R


def copy_corners(t: Tile, q_in, direction, out=None):
    """copy_corners_x/y_stencil_defn (corners.py:306-422): returns a copy of
    q_in with the 3x3 corner blocks filled from the tile edges so that the
    field can be differenced in x (direction 'x') or y ('y')."""
    rules = _copy_rules_x(t) if direction == "x" else _copy_rules_y(t)
    res = np.array(q_in if out is None else out, copy=True)
    for (i, j), (di, dj) in rules:
        if 0 <= i < t.m and 0 <= j < t.m:
            res[i, j] = q_in[i + di, j + dj]
    return res
