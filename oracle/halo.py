"""Cubed-sphere halo exchange for the oracle (six tiles in one array).

Restates the behaviour of fv3gfs-util's halo updaters that the reference's
AcousticDynamics uses (dyn_core.py:216-286; fv3gfs-util is not part of the
reference checkout, so this is pinned by the analytic-field test, not by
golden data).  Implemented with whole edge slabs: the halo strip outside an
edge of one tile is the interior strip inside the matching edge of the
neighbouring tile, reversed along the edge where the two tiles run in
opposite directions, and for vectors with components exchanged and signs
flipped as the tile orientation requires.  The 3x3 corner blocks are not
written.

Tile connectivity (0-based): even t: E->(t+1, W), N->(t+2, W, reversed),
W->(t-2, N, reversed), S->(t-1, N); odd t: E->(t+2, S, reversed),
N->(t+1, S), W->(t-1, E), S->(t-2, E, reversed).
"""
import numpy as np


def _neighbor(t, edge):
    if t % 2 == 0:
        return {"E": ((t + 1) % 6, "W", False), "N": ((t + 2) % 6, "W", True),
                "W": ((t - 2) % 6, "N", True), "S": ((t - 1) % 6, "N", False)}[edge]
    return {"E": ((t + 2) % 6, "S", True), "N": ((t + 1) % 6, "S", False),
            "W": ((t - 1) % 6, "E", False), "S": ((t - 2) % 6, "E", True)}[edge]


class HaloExchange:
    def __init__(self, n, h=3):
        self.n, self.h = n, h

    # --------------------------------------------------------------- slabs
    def _halo_index(self, edge, depth, along, sx, sy):
        """Storage (i, j) of our halo point ``depth`` cells outside ``edge``
        (0 = adjacent) at position ``along`` on the edge."""
        n, h = self.n, self.h
        if edge == "W":
            return h - 1 - depth, h + along
        if edge == "E":
            return h + n + (1 - sx) + depth, h + along
        if edge == "S":
            return h + along, h - 1 - depth
        return h + along, h + n + (1 - sy) + depth

    def _interior_index(self, edge, depth, along, sx, sy):
        """Storage (i, j) of the neighbour's point ``depth`` cells inside
        ``edge`` (0 = first point off the edge line)."""
        n, h = self.n, self.h
        if edge == "W":
            return h + (1 - sx) + depth, h + along
        if edge == "E":
            return h + n - 1 - depth, h + along
        if edge == "S":
            return h + along, h + (1 - sy) + depth
        return h + along, h + n - 1 - depth

    def _edge_points(self, edge, sx, sy, nh):
        n = self.n
        along_stagger = sy if edge in ("W", "E") else sx
        L = n if along_stagger == 1 else n + 1
        return [(d, a) for d in range(nh) for a in range(L)], L

    # --------------------------------------------------------------- exchanges
    def _exchange(self, fields, staggers, vector, nh, nk):
        """fields: list of 6-tile arrays; staggers: list of (sx, sy); for a
        vector, fields = [x component, y component]."""
        src = [np.array(f[..., :nk], copy=True) for f in fields]
        for t in range(6):
            for edge in ("W", "E", "S", "N"):
                t2, e2, rev = _neighbor(t, edge)
                perpendicular = (edge in ("W", "E")) != (e2 in ("W", "E"))
                for c, f in enumerate(fields):
                    sx, sy = staggers[c]
                    pts, L = self._edge_points(edge, sx, sy, nh)
                    if vector:
                        # which neighbour component and sign give ours
                        normal_ours = 0 if edge in ("W", "E") else 1
                        if c == normal_ours:
                            c2 = 0 if e2 in ("W", "E") else 1
                            out_sign = -1 if edge in ("W", "S") else 1
                            in_sign = 1 if e2 in ("W", "S") else -1
                            sign = out_sign * in_sign
                        else:
                            c2 = 1 if e2 in ("W", "E") else 0
                            sign = -1 if rev else 1
                    else:
                        c2, sign = c, 1
                    sx2, sy2 = (sy, sx) if perpendicular else (sx, sy)
                    for d, a in pts:
                        a2 = (L - 1 - a) if rev else a
                        i, j = self._halo_index(edge, d, a, sx, sy)
                        i2, j2 = self._interior_index(e2, d, a2, sx2, sy2)
                        f[t, i, j, :nk] = sign * src[c2][t2, i2, j2, :nk]

    def _nk(self, f, nk):
        return f.shape[-1] if nk is None else nk

    def scalar(self, *fields, n_halo=None, nk=None):
        """Cell-centred scalars (X, Y dims)."""
        nh = self.h if n_halo is None else n_halo
        for f in fields:
            self._exchange([f], [(1, 1)], False, nh, self._nk(f, nk))

    def scalar_corner(self, *fields, n_halo=None, nk=None):
        """Cell-corner scalars (X_INTERFACE, Y_INTERFACE dims)."""
        nh = self.h if n_halo is None else n_halo
        for f in fields:
            self._exchange([f], [(0, 0)], False, nh, self._nk(f, nk))

    def vector_d(self, u, v, nk=None):
        """D-grid winds: u on (X, Y_INTERFACE), v on (X_INTERFACE, Y)."""
        self._exchange([u, v], [(1, 0), (0, 1)], True, self.h, self._nk(u, nk))

    def vector_c(self, uc, vc, nk=None):
        """C-grid winds: uc on (X_INTERFACE, Y), vc on (X, Y_INTERFACE)."""
        self._exchange([uc, vc], [(0, 1), (1, 0)], True, self.h, self._nk(uc, nk))

    def sync_vector_interfaces(self, u, v, nk=None):
        """synchronize_vector_interfaces for D-grid winds: each tile's u on its
        south edge line and v on its west edge line overwrite the shared edge
        line of the neighbouring tile (rotated as needed)."""
        n, h = self.n, self.h
        nk = self._nk(u, nk)
        src = (np.array(u[..., :nk], copy=True), np.array(v[..., :nk], copy=True))
        dst = (u, v)
        for t in range(6):
            for edge, comp in (("S", 0), ("W", 1)):
                t2, e2, rev = _neighbor(t, edge)
                comp2 = 0 if e2 in ("S", "N") else 1
                sign = -1 if rev else 1
                for a in range(n):
                    a2 = n - 1 - a if rev else a
                    si, sj = (h + a, h) if edge == "S" else (h, h + a)
                    if e2 == "W":
                        di, dj = h, h + a2
                    elif e2 == "E":
                        di, dj = h + n, h + a2
                    elif e2 == "S":
                        di, dj = h + a2, h
                    else:
                        di, dj = h + a2, h + n
                    dst[comp2][t2, di, dj, :nk] = sign * src[comp][t, si, sj, :nk]
