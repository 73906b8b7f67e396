"""Cubed-sphere tile connectivity and halo gather tables.

All six tiles of the cube live in one array ``[6, ni+2h+1, nj+2h+1, nz+1]``
(Python index order i, j, k).  A halo exchange is therefore a gather inside
device memory: every halo point of tile ``t`` copies (and, for vectors,
rotates) one compute-domain value of a neighbouring tile.  This module builds
the gather tables on the host once; ``fv3core_b200.halo`` uploads them and
runs the gather kernel.

Tile numbering and edge connectivity follow the FV3 cube (0-based tiles):

* even tile t: east -> t+1 (aligned), north -> t+2 (rotated: our north edge is
  its west edge, running the other way), west -> t-2 (its north edge,
  reversed), south -> t-1 (its north edge, aligned);
* odd tile t: east -> t+2 (its south edge, reversed), north -> t+1 (its south
  edge, aligned), west -> t-1 (its east edge, aligned), south -> t-2 (its
  east edge, reversed).

This is the connectivity of fv3gfs-util's ``TilePartitioner`` that the
reference's halo updaters use (``fv3core/stencils/dyn_core.py:216-286`` builds
them; fv3gfs-util itself is not part of the reference checkout).  The 3x3
corner blocks beyond two tile edges have no neighbour and are not written,
as in fv3gfs-util; the stencils fill them themselves (``utils/corners.py``).

Positions are handled in "doubled" index space: along each axis a cell
centre i is at 2i+1 and an interface i at 2i, both relative to the first
compute cell.  A point outside edge E of tile t at depth d maps to depth d
inside the matching edge E' of the neighbour, at the same (or mirrored)
position along the edge.
"""
import numpy as np

WEST, EAST, SOUTH, NORTH = "W", "E", "S", "N"


def edge_neighbor(tile, edge):
    """Return (neighbour tile, neighbour edge, reversed) for ``edge`` of ``tile``."""
    if tile % 2 == 0:
        table = {
            EAST: ((tile + 1) % 6, WEST, False),
            NORTH: ((tile + 2) % 6, WEST, True),
            WEST: ((tile - 2) % 6, NORTH, True),
            SOUTH: ((tile - 1) % 6, NORTH, False),
        }
    else:
        table = {
            EAST: ((tile + 2) % 6, SOUTH, True),
            NORTH: ((tile + 1) % 6, SOUTH, False),
            WEST: ((tile - 1) % 6, EAST, False),
            SOUTH: ((tile - 2) % 6, EAST, True),
        }
    return table[edge]


# unit directions as (axis, sign): axis 0 = x (i), 1 = y (j)
_OUTWARD = {EAST: (0, 1), WEST: (0, -1), NORTH: (1, 1), SOUTH: (1, -1)}
_INWARD = {WEST: (0, 1), EAST: (0, -1), SOUTH: (1, 1), NORTH: (1, -1)}
_ALONG = {WEST: (1, 1), EAST: (1, 1), SOUTH: (0, 1), NORTH: (0, 1)}


def map_point(n, tile, X, Y):
    """Map a doubled-index halo point (X, Y) of ``tile`` (exactly one coordinate
    outside [0, 2n]) to (tile', X', Y', dirmap) where ``dirmap[a] = (a', s)``
    says that our unit vector along axis a is s times the neighbour's unit
    vector along axis a'."""
    nn = 2 * n
    if X > nn:
        edge, d, s = EAST, X - nn, Y
    elif X < 0:
        edge, d, s = WEST, -X, Y
    elif Y > nn:
        edge, d, s = NORTH, Y - nn, X
    elif Y < 0:
        edge, d, s = SOUTH, -Y, X
    else:
        raise ValueError("point is not in an edge halo")
    t2, e2, rev = edge_neighbor(tile, edge)
    s2 = nn - s if rev else s
    if e2 == WEST:
        X2, Y2 = d, s2
    elif e2 == EAST:
        X2, Y2 = nn - d, s2
    elif e2 == SOUTH:
        X2, Y2 = s2, d
    else:
        X2, Y2 = s2, nn - d
    # direction map
    out_axis, out_sign = _OUTWARD[edge]
    in_axis, in_sign = _INWARD[e2]
    al_axis, al_sign = _ALONG[edge]
    al2_axis, al2_sign = _ALONG[e2]
    if rev:
        al2_sign = -al2_sign
    dirmap = {}
    # our outward normal == neighbour inward normal
    dirmap[out_axis] = (in_axis, out_sign * in_sign)
    # our along-edge direction == neighbour along-edge direction (maybe reversed)
    dirmap[al_axis] = (al2_axis, al_sign * al2_sign)
    return t2, X2, Y2, dirmap


def _compute_range(n, stagger):
    """Compute-domain offsets (relative to the first compute cell) for a
    staggering: 1 = cell centre (0..n-1), 0 = interface (0..n)."""
    return range(n) if stagger == 1 else range(n + 1)


def _halo_offsets(n, stagger, n_halo):
    lo = list(range(-n_halo, 0))
    hi = list(range(n, n + n_halo)) if stagger == 1 else list(range(n + 1, n + 1 + n_halo))
    return lo, hi


def halo_points(n, sx, sy, n_halo):
    """Yield (a, b) compute-relative offsets of every edge-halo point (corner
    blocks excluded) of a field with staggering (sx, sy)."""
    xs = list(_compute_range(n, sx))
    ys = list(_compute_range(n, sy))
    xlo, xhi = _halo_offsets(n, sx, n_halo)
    ylo, yhi = _halo_offsets(n, sy, n_halo)
    for a in xlo + xhi:
        for b in ys:
            yield a, b
    for b in ylo + yhi:
        for a in xs:
            yield a, b


def scalar_table(n, h, sx, sy, n_halo):
    """Gather table for a scalar field: int64 array [m, 6] with columns
    (dst_tile, dst_i, dst_j, src_tile, src_i, src_j) in storage indices."""
    rows = []
    for t in range(6):
        for a, b in halo_points(n, sx, sy, n_halo):
            X, Y = 2 * a + sx, 2 * b + sy
            t2, X2, Y2, dirmap = map_point(n, t, X, Y)
            swap = dirmap[0][0] == 1
            sx2, sy2 = (sy, sx) if swap else (sx, sy)
            if swap and sx != sy:
                raise ValueError("scalar staggering changes across a rotated edge")
            a2 = (X2 - sx2) // 2
            b2 = (Y2 - sy2) // 2
            assert 2 * a2 + sx2 == X2 and 2 * b2 + sy2 == Y2
            rows.append((t, a + h, b + h, t2, a2 + h, b2 + h))
    return np.asarray(rows, dtype=np.int64)


def scalar_table_any(n, h, s, n_halo):
    """Scalar table for centre (s=1) or corner (s=0) fields, where staggering is
    the same on both axes and so survives tile rotation."""
    return scalar_table(n, h, s, s, n_halo)


def vector_tables(n, h, x_stagger, y_stagger, n_halo):
    """Gather tables for a vector whose x component has staggering
    ``x_stagger`` and y component ``y_stagger`` (each a (sx, sy) pair; the y
    component's is the x component's transposed, as for D-grid (u, v) or
    C-grid (uc, vc)).

    Returns two int64 arrays (for the x and y component fields), each
    [m, 8] with columns (dst_tile, dst_i, dst_j, src_tile, src_i, src_j,
    src_component, sign); ``src_component`` 0 = x field, 1 = y field.
    """
    out = []
    for comp, (sx, sy) in enumerate((x_stagger, y_stagger)):
        rows = []
        for t in range(6):
            for a, b in halo_points(n, sx, sy, n_halo):
                X, Y = 2 * a + sx, 2 * b + sy
                t2, X2, Y2, dirmap = map_point(n, t, X, Y)
                ax2, sgn = dirmap[comp]
                st2 = x_stagger if ax2 == 0 else y_stagger
                a2 = (X2 - st2[0]) // 2
                b2 = (Y2 - st2[1]) // 2
                assert 2 * a2 + st2[0] == X2 and 2 * b2 + st2[1] == Y2, (t, a, b, comp)
                rows.append((t, a + h, b + h, t2, a2 + h, b2 + h, ax2, sgn))
        out.append(np.asarray(rows, dtype=np.int64))
    return out


def interface_sync_tables(n, h):
    """Tables for ``synchronize_vector_interfaces`` on D-grid winds.

    The values of u on each tile's south edge line (j interface 0) and of v on
    its west edge line (i interface 0) are copied, rotated as needed, over the
    shared edge line of the neighbouring tile, so both tiles hold identical
    values there.  Returns a list of rows (dst_tile, dst_comp, dst_i, dst_j,
    src_tile, src_comp, src_i, src_j, sign); comp 0 = u, 1 = v.
    """
    rows = []
    nn = 2 * n
    for t in range(6):
        # u on the south edge line: positions X = 2a+1, Y = 0; direction +x
        for edge, comp in ((SOUTH, 0), (WEST, 1)):
            t2, e2, rev = edge_neighbor(t, edge)
            for a in range(n):
                s = 2 * a + 1
                s2 = nn - s if rev else s
                if e2 == WEST:
                    X2, Y2 = 0, s2
                elif e2 == EAST:
                    X2, Y2 = nn, s2
                elif e2 == SOUTH:
                    X2, Y2 = s2, 0
                else:
                    X2, Y2 = s2, nn
                al_axis, al_sign = _ALONG[edge]
                al2_axis, al2_sign = _ALONG[e2]
                if rev:
                    al2_sign = -al2_sign
                comp2 = al2_axis
                sign = al_sign * al2_sign
                # source position in our tile
                if edge == SOUTH:
                    si, sj = a, 0
                else:
                    si, sj = 0, a
                # destination in the neighbour: stagger of comp2 is (1,0) for u, (0,1) for v
                st2 = (1, 0) if comp2 == 0 else (0, 1)
                di = (X2 - st2[0]) // 2
                dj = (Y2 - st2[1]) // 2
                rows.append((t2, comp2, di + h, dj + h, t, comp, si + h, sj + h, sign))
    return np.asarray(rows, dtype=np.int64)


def apply_scalar_table(arr, table):
    """Host-side gather: ``arr`` is [6, I, J, ...]; fills the table's halo points."""
    d = table
    arr[d[:, 0], d[:, 1], d[:, 2]] = arr[d[:, 3], d[:, 4], d[:, 5]]


def apply_vector_tables(ux, uy, tables):
    """Host-side vector gather with rotation (see ``vector_tables``)."""
    src = (ux.copy(), uy.copy())
    for dst, d in zip((ux, uy), tables):
        vals = np.where(
            (d[:, 6] == 0).reshape((-1,) + (1,) * (ux.ndim - 3)),
            src[0][d[:, 3], d[:, 4], d[:, 5]],
            src[1][d[:, 3], d[:, 4], d[:, 5]],
        )
        dst[d[:, 0], d[:, 1], d[:, 2]] = vals * d[:, 7].reshape((-1,) + (1,) * (ux.ndim - 3))
