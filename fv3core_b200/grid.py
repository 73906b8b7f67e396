"""Equiangular gnomonic cubed-sphere grid and the metric terms the acoustic
substep reads.

This is host-side set-up (numpy, FP64), run once per resolution.  It plays
the role of the reference's ``MetricTerms`` (``fv3core/grid/generation.py``)
and ``DampingCoefficients``/``GridData`` containers (``fv3core/utils/grid.py``
475-799): it produces the ~40 two-dimensional fields the stencils consume,
for all six tiles at once, with halos.

Construction (our own, from the standard FV3 cube geometry):

* Cell corners of each face are the gnomonic projection of a lattice of
  face coordinates (``face_coordinates``): by default equiangular (alpha,
  beta on [-pi/4, pi/4]^2); ``lattice="equidistant"`` gives the reference's
  gnomonic_ed (grid_type 0), whose edge points are equally spaced along the
  edges.  Faces are oriented so that the tile connectivity is the FV3 one in
  ``halo_map`` (tile 0 as the reference's first tile).
* Halo corner points come from the neighbouring tile through the same halo
  gather as the dynamics (as the reference fills them with a halo update);
  the 3x3 blocks beyond two tile edges, which have no neighbour, extend the
  local equiangular lattice.
* Lengths are great-circle distances times the Earth radius, areas are
  spherical-quadrilateral excess times radius squared, angles are taken
  between great-circle tangents.  Metric combinations (cosa_u, rsin2,
  del6_u, divg_u, edge factors ...) follow the FV3 definitions cited per
  field below.
"""
import numpy as np

from . import constants
from .halo_map import WEST, EAST, SOUTH, NORTH, edge_neighbor, map_point

N_TILES = 6

# face frames (centre, local x axis, local y axis), right handed
_FACES = [
    ((1, 0, 0), (0, 1, 0), (0, 0, 1)),
    ((0, 1, 0), (-1, 0, 0), (0, 0, 1)),
    ((0, 0, 1), (-1, 0, 0), (0, -1, 0)),
    ((-1, 0, 0), (0, 0, -1), (0, -1, 0)),
    ((0, -1, 0), (0, 0, -1), (1, 0, 0)),
    ((0, 0, -1), (0, 1, 0), (1, 0, 0)),
]


def _face_points(tile, ua, ub):
    """Unit vectors c + ua ex + ub ey of face ``tile`` for face coordinates
    ua, ub (1 at the face's edges)."""
    c, ex, ey = (np.asarray(v, dtype=np.float64) for v in _FACES[tile])
    p = (
        c[None, None, :]
        + ua[:, :, None] * ex[None, None, :]
        + ub[:, :, None] * ey[None, None, :]
    )
    return p / np.linalg.norm(p, axis=-1, keepdims=True)


LATTICES = ("equiangular", "equidistant")


def face_coordinates(n, halo, lattice="equiangular"):
    """Face coordinate (1 at the face's edges) of the lattice lines -halo ..
    n + halo.  ``equiangular``: tan of equally spaced angles from the face
    centre, -pi/4 .. pi/4 over the face.  ``equidistant``: the reference's
    gnomonic_ed (grid_type 0, fv3core/grid/global_setup.py:42-85), whose
    edge points are equally spaced along the edge great circles (latitudes
    -a .. a along the edge meridian, a = asin(1/sqrt(3))); on the face plane
    that is sqrt(2) tan of those latitudes.  The halo lines continue the same
    spacing."""
    idx = np.arange(-halo, n + halo + 1)
    if lattice == "equiangular":
        dal = 0.5 * np.pi / n
        return np.tan(-0.25 * np.pi + idx * dal)
    if lattice == "equidistant":
        alpha = np.arcsin(3 ** -0.5)
        dely = 2.0 * alpha / n
        return np.sqrt(2.0) * np.tan(-alpha + idx * dely)
    raise ValueError(f"lattice must be one of {LATTICES}, got {lattice!r}")


def _normalize(p):
    return p / np.linalg.norm(p, axis=-1, keepdims=True)


def _gc_dist(p, q):
    """Great-circle angle between unit vectors (robust atan2 form)."""
    cr = np.linalg.norm(np.cross(p, q), axis=-1)
    dt = np.sum(p * q, axis=-1)
    return np.arctan2(cr, dt)


def _tangent(p, q):
    """Unit tangent at p of the great circle towards q."""
    t = q - np.sum(q * p, axis=-1, keepdims=True) * p
    norm = np.linalg.norm(t, axis=-1, keepdims=True)
    # Where q coincides with p (the halo points that fold onto a cube vertex)
    # the tangent is undefined: those points hold NaN, set explicitly.
    defined = norm > 0.0
    return np.where(defined, t / np.where(defined, norm, 1.0), np.nan)


def _cos_angle(p, q1, q2):
    return np.sum(_tangent(p, q1) * _tangent(p, q2), axis=-1)


def _tri_area(a, b, c):
    """Spherical excess of a triangle (L'Huilier via the vector formula)."""
    num = np.abs(np.sum(a * np.cross(b, c), axis=-1))
    den = 1.0 + np.sum(a * b, axis=-1) + np.sum(b * c, axis=-1) + np.sum(c * a, axis=-1)
    return 2.0 * np.arctan2(num, den)


def _quad_area(p1, p2, p3, p4):
    return _tri_area(p1, p2, p3) + _tri_area(p1, p3, p4)


def _lonlat(p):
    lon = np.arctan2(p[..., 1], p[..., 0])
    lon = np.where(lon < 0, lon + 2 * np.pi, lon)
    lat = np.arcsin(np.clip(p[..., 2], -1.0, 1.0))
    return lon, lat


class CubedSphereGrid:
    """Metric terms for all six tiles, each field shaped like the reference's
    ``max_shape`` (``stencil.py:357-367``): ``[6, n+2h+1, n+2h+1]`` with the
    compute domain starting at index ``h``."""

    def __init__(self, n, halo=3, radius=constants.RADIUS, lattice="equiangular"):
        self.n = n
        self.halo = h = halo
        self.radius = radius
        self.lattice = lattice
        m = n + 2 * h + 1
        self.shape2d = (N_TILES, m, m)
        self._build_corners()
        self._build_metrics()

    # ------------------------------------------------------------------ corners
    def _build_corners(self):
        n, h = self.n, self.halo
        m = n + 2 * h + 1
        u1 = face_coordinates(n, h, self.lattice)
        ua, ub = np.meshgrid(u1, u1, indexing="ij")
        P = np.empty((N_TILES, m, m, 3))
        for t in range(N_TILES):
            P[t] = _face_points(t, ua, ub)
        # snap each point to its exact cube-symmetric value: rebuild the halo
        # edge ring from the neighbour tiles so that shared points coincide
        for t in range(N_TILES):
            for a in range(-h, n + h + 1):
                for b in range(-h, n + h + 1):
                    inx = 0 <= a <= n
                    iny = 0 <= b <= n
                    if inx == iny:
                        continue  # compute points, or corner blocks (keep extension)
                    t2, X2, Y2, _ = map_point(n, t, 2 * a, 2 * b)
                    P[t, a + h, b + h] = P[t2, X2 // 2 + h, Y2 // 2 + h]
        self.corners = P
        self.lon_b, self.lat_b = _lonlat(P)

    # ------------------------------------------------------------------ metrics
    def _build_metrics(self):
        n, h, R = self.n, self.halo, self.radius
        P = self.corners
        m = n + 2 * h + 1
        z = np.zeros(self.shape2d)

        def pad2(arr):
            out = np.zeros(self.shape2d)
            out[:, : arr.shape[1], : arr.shape[2]] = arr
            return out

        p00 = P[:, :-1, :-1]
        p10 = P[:, 1:, :-1]
        p01 = P[:, :-1, 1:]
        p11 = P[:, 1:, 1:]
        # cell centres (A grid): normalised sum of the four corners
        C = _normalize(p00 + p10 + p01 + p11)  # [6, m-1, m-1]
        self.centers = C
        lon_a, lat_a = _lonlat(C)
        self.lon_a = pad2(lon_a)
        self.lat_a = pad2(lat_a)
        # D-grid edge lengths
        dx = pad2(_gc_dist(P[:, :-1, :], P[:, 1:, :]) * R)  # u points: [i, j] between P[i,j],P[i+1,j]
        dy = pad2(_gc_dist(P[:, :, :-1], P[:, :, 1:]) * R)
        # edge midpoints
        mw = _normalize(p00 + p01)  # west edge midpoint of cell (i,j)
        me = _normalize(p10 + p11)
        ms = _normalize(p00 + p10)
        mn = _normalize(p01 + p11)
        dxa = pad2(_gc_dist(mw, me) * R)
        dya = pad2(_gc_dist(ms, mn) * R)
        # C-grid distances between centres
        dxc = z.copy()
        dxc[:, 1 : m - 1, : m - 1] = _gc_dist(C[:, :-1, :], C[:, 1:, :]) * R
        dxc[:, 0, :] = dxc[:, 1, :]
        dyc = z.copy()
        dyc[:, : m - 1, 1 : m - 1] = _gc_dist(C[:, :, :-1], C[:, :, 1:]) * R
        dyc[:, :, 0] = dyc[:, :, 1]
        area = pad2(_quad_area(p00, p10, p11, p01) * R * R)
        area_c = z.copy()
        area_c[:, 1 : m - 1, 1 : m - 1] = (
            _quad_area(C[:, :-1, :-1], C[:, 1:, :-1], C[:, 1:, 1:], C[:, :-1, 1:]) * R * R
        )
        area_c[:, 0, :] = area_c[:, 1, :]
        area_c[:, :, 0] = area_c[:, :, 1]

        # angles at edge midpoints and centres (FV3 cos_sg/sin_sg 1..5):
        # 1 west-edge midpoint, 2 south, 3 east, 4 north, 5 centre; in each the
        # angle between the local x and y directions.
        cos_sg = {}
        cos_sg[1] = _cos_angle(mw, C, p01)
        cos_sg[2] = _cos_angle(ms, p10, C)
        cos_sg[3] = _cos_angle(me, 2 * me - C, p11)  # x direction continues outward
        cos_sg[4] = _cos_angle(mn, p11, 2 * mn - C)
        cos_sg[5] = _cos_angle(C, me, mn)
        sin_sg = {k: np.minimum(1.0, np.sqrt(np.maximum(0.0, 1.0 - v * v))) for k, v in cos_sg.items()}
        self._corner_fix(cos_sg, sin_sg)
        for k in range(1, 6):
            setattr(self, f"cos_sg{k}", pad2(cos_sg[k]))
            setattr(self, f"sin_sg{k}", pad2(sin_sg[k]))
        # corner angle (B grid): between the grid lines through the corner
        cfwd = _cos_angle(P[:, 1:-1, 1:-1], P[:, 2:, 1:-1], P[:, 1:-1, 2:])
        cbwd = _cos_angle(
            P[:, 1:-1, 1:-1], 2 * P[:, 1:-1, 1:-1] - P[:, :-2, 1:-1], 2 * P[:, 1:-1, 1:-1] - P[:, 1:-1, :-2]
        )
        cosa = z.copy()
        cosa[:, 1:-1, 1:-1] = 0.5 * (cfwd + cbwd)
        sina = np.sqrt(np.maximum(1.0 - cosa * cosa, 0.0))
        tiny = 1.0e-30

        # FV3 combinations (fv_grid_tools init_grid)
        cosa_u = z.copy()
        sina_u = np.ones(self.shape2d)
        cosa_u[:, 1:, :] = 0.5 * (self.cos_sg3[:, :-1, :] + self.cos_sg1[:, 1:, :])
        sina_u[:, 1:, :] = 0.5 * (self.sin_sg3[:, :-1, :] + self.sin_sg1[:, 1:, :])
        cosa_v = z.copy()
        sina_v = np.ones(self.shape2d)
        cosa_v[:, :, 1:] = 0.5 * (self.cos_sg4[:, :, :-1] + self.cos_sg2[:, :, 1:])
        sina_v[:, :, 1:] = 0.5 * (self.sin_sg4[:, :, :-1] + self.sin_sg2[:, :, 1:])
        # on tile edges the two sides belong to different tiles; use the inner cell
        for t in range(N_TILES):
            pass
        rsin_u = 1.0 / np.maximum(tiny, sina_u**2)
        rsin_v = 1.0 / np.maximum(tiny, sina_v**2)
        cosa_s = self.cos_sg5.copy()
        rsin2 = 1.0 / np.maximum(tiny, self.sin_sg5**2)
        rsina = 1.0 / np.maximum(tiny, sina**2)

        # fill unset rows/columns (array padding) with benign values
        for arr, val in ((dx, None), (dy, None), (dxa, None), (dya, None), (area, None)):
            pass
        self.dx, self.dy, self.dxa, self.dya = dx, dy, dxa, dya
        self.dxc, self.dyc = dxc, dyc
        self.area, self.area_c = area, area_c
        self.cosa, self.sina, self.rsina = cosa, sina, rsina
        self.cosa_u, self.sina_u, self.rsin_u = cosa_u, sina_u, rsin_u
        self.cosa_v, self.sina_v, self.rsin_v = cosa_v, sina_v, rsin_v
        self.cosa_s, self.rsin2 = cosa_s, rsin2
        with np.errstate(divide="ignore", invalid="ignore"):
            self.rarea = np.where(area > 0, 1.0 / np.where(area > 0, area, 1.0), 0.0)
            self.rarea_c = np.where(area_c > 0, 1.0 / np.where(area_c > 0, area_c, 1.0), 0.0)
            self.rdx = np.where(dx > 0, 1.0 / np.where(dx > 0, dx, 1.0), 0.0)
            self.rdy = np.where(dy > 0, 1.0 / np.where(dy > 0, dy, 1.0), 0.0)
            self.rdxa = np.where(dxa > 0, 1.0 / np.where(dxa > 0, dxa, 1.0), 0.0)
            self.rdya = np.where(dya > 0, 1.0 / np.where(dya > 0, dya, 1.0), 0.0)
            self.rdxc = np.where(dxc > 0, 1.0 / np.where(dxc > 0, dxc, 1.0), 0.0)
            self.rdyc = np.where(dyc > 0, 1.0 / np.where(dyc > 0, dyc, 1.0), 0.0)
            # damping coefficients (fv3core/grid/geometry.py:514-585)
            self.divg_u = np.where(dx > 0, sina_v * dyc / np.where(dx > 0, dx, 1.0), 0.0)
            self.del6_u = np.where(dyc > 0, sina_v * dx / np.where(dyc > 0, dyc, 1.0), 0.0)
            self.divg_v = np.where(dy > 0, sina_u * dxc / np.where(dy > 0, dy, 1.0), 0.0)
            self.del6_v = np.where(dxc > 0, sina_u * dy / np.where(dxc > 0, dxc, 1.0), 0.0)
        # tile-edge rows use the average of the sine on the two sides (same file)
        hs, he = h, h + n
        s_b = 0.5 * (self.sin_sg2[:, :, hs] + self.sin_sg4[:, :, hs - 1])
        s_t = 0.5 * (self.sin_sg2[:, :, he] + self.sin_sg4[:, :, he - 1])
        self.divg_u[:, :, hs] = s_b * dyc[:, :, hs] / np.where(dx[:, :, hs] > 0, dx[:, :, hs], 1)
        self.del6_u[:, :, hs] = s_b * dx[:, :, hs] / np.where(dyc[:, :, hs] > 0, dyc[:, :, hs], 1)
        self.divg_u[:, :, he] = s_t * dyc[:, :, he] / np.where(dx[:, :, he] > 0, dx[:, :, he], 1)
        self.del6_u[:, :, he] = s_t * dx[:, :, he] / np.where(dyc[:, :, he] > 0, dyc[:, :, he], 1)
        s_l = 0.5 * (self.sin_sg1[:, hs, :] + self.sin_sg3[:, hs - 1, :])
        s_r = 0.5 * (self.sin_sg1[:, he, :] + self.sin_sg3[:, he - 1, :])
        self.divg_v[:, hs, :] = s_l * dxc[:, hs, :] / np.where(dy[:, hs, :] > 0, dy[:, hs, :], 1)
        self.del6_v[:, hs, :] = s_l * dy[:, hs, :] / np.where(dxc[:, hs, :] > 0, dxc[:, hs, :], 1)
        self.divg_v[:, he, :] = s_r * dxc[:, he, :] / np.where(dy[:, he, :] > 0, dy[:, he, :], 1)
        self.del6_v[:, he, :] = s_r * dy[:, he, :] / np.where(dxc[:, he, :] > 0, dxc[:, he, :], 1)

        # Coriolis on corners (fC) and centres (f0)
        om2 = 2.0 * constants.OMEGA
        self.fC = om2 * np.sin(self.lat_b)
        self.f0 = pad2(om2 * np.sin(lat_a))
        # A/B grid lon-lat (agrid1/2, bgrid1/2 in a2b_ord4)
        self.agrid1, self.agrid2 = self.lon_a, self.lat_a
        self.bgrid1, self.bgrid2 = self.lon_b, self.lat_b
        # A->B edge interpolation factors (fv3core/grid/geometry.py:604-714)
        self.edge_w, self.edge_e, self.edge_s, self.edge_n = self._edge_factors(C)
        self.a2b_extrap = self._a2b_extrap_ratios()
        self._cubed_to_latlon(C, me, mn)
        # minimum areas over the six compute domains
        self.da_min = float(area[:, hs:he, hs:he].min())
        self.da_max = float(area[:, hs:he, hs:he].max())
        self.da_min_c = float(area_c[:, hs : he + 1, hs : he + 1].min())
        self.da_max_c = float(area_c[:, hs : he + 1, hs : he + 1].max())

    # (near, far) A-grid offsets of the three extrapolations at each tile
    # corner of a2b_ord4 (a2b_ord4.py:60-235); the corners are, in order, the
    # B-grid points (is, js), (ie+1, js), (ie+1, je+1), (is, je+1), whose
    # reference stencils are _sw, _nw, _ne, _se
    A2B_CORNER_OFFSETS = (
        (((0, 0), (1, 1)), ((-1, 0), (-2, 1)), ((0, -1), (1, -2))),
        (((-1, 0), (-2, 1)), ((-1, -1), (-2, -2)), ((0, 0), (1, 1))),
        (((-1, -1), (-2, -2)), ((0, -1), (1, -2)), ((-1, 0), (-2, 1))),
        (((0, -1), (1, -2)), ((-1, -1), (-2, -2)), ((0, 0), (1, 1))),
    )

    def _a2b_extrap_ratios(self):
        """x1 / (x2 - x1) of each cube-corner extrapolation of a2b_ord4
        (extrap_corner, a2b_ord4.py:45-57): x1, x2 are the great-circle
        distances (a2b_ord4.py:38-41) from the B-grid corner to the near and
        far A-grid points.  They depend on the grid only, so they are computed
        once here.  Returns [6, 4, 3] in the order of A2B_CORNER_OFFSETS."""
        h, n = self.halo, self.n
        s, e = h, h + n - 1
        corners = ((s, s), (e + 1, s), (e + 1, e + 1), (s, e + 1))

        def gcd(p1a, p1b, p2a, p2b):
            tb = np.sin((p1b - p2b) / 2.0) ** 2.0
            ta = np.sin((p1a - p2a) / 2.0) ** 2.0
            return np.arcsin(np.sqrt(tb + np.cos(p1b) * np.cos(p2b) * ta)) * 2.0

        out = np.zeros((6, 4, 3))
        for c, (i, j) in enumerate(corners):
            b1, b2 = self.bgrid1[:, i, j], self.bgrid2[:, i, j]
            for m, ((di1, dj1), (di2, dj2)) in enumerate(self.A2B_CORNER_OFFSETS[c]):
                x1 = gcd(self.agrid1[:, i + di1, j + dj1], self.agrid2[:, i + di1, j + dj1], b1, b2)
                x2 = gcd(self.agrid1[:, i + di2, j + dj2], self.agrid2[:, i + di2, j + dj2], b1, b2)
                out[:, c, m] = x1 / (x2 - x1)
        return out

    def _corner_fix(self, cos_sg, sin_sg):
        """Angles in the 3x3 cube-corner halo blocks, which have no cell of
        their own on the sphere, follow FV3's convention
        (fv3core/grid/geometry.py:430-512): the block is filled with
        sin = 1e-8, cos = 1e8, then the edge angles facing the adjacent edge
        halos are rotated in from those halo cells."""
        h = self.halo
        N = cos_sg[1].shape[1]  # cell-centred extent n + 2h
        for arrs, fill in ((sin_sg, 1.0e-8), (cos_sg, 1.0e8)):
            for k in range(1, 6):
                a = arrs[k]
                a[:, :h, :h] = fill
                a[:, :h, N - h :] = fill
                a[:, N - h :, :h] = fill
                a[:, N - h :, N - h :] = fill
            sg1, sg2, sg3, sg4 = arrs[1], arrs[2], arrs[3], arrs[4]
            for a in range(h):
                # south-west
                sg3[:, h - 1, a] = sg2[:, a, h]
                sg4[:, a, h - 1] = sg1[:, h, a]
                # north-west
                sg2[:, a, N - h] = sg1[:, h, N - 1 - a]
                sg3[:, h - 1, N - 1 - a] = sg4[:, a, N - 1 - h]
                # south-east
                sg1[:, N - h, a] = sg2[:, N - 1 - a, h]
                sg4[:, N - 1 - a, h - 1] = sg3[:, N - 1 - h, a]
                # north-east
                sg1[:, N - h, N - 1 - a] = sg4[:, N - 1 - a, N - 1 - h]
                sg2[:, N - 1 - a, N - h] = sg3[:, N - 1 - h, N - 1 - a]

    def _edge_factors(self, C):
        """1-D A->B interpolation weights along the four tile edges; entries
        0 and n (cube corners) stay at the reference's fill value 1e8."""
        n, h = self.n, self.halo
        P = self.corners
        big = 1.0e8
        out = []
        for edge in (WEST, EAST, SOUTH, NORTH):
            e = np.full((N_TILES, n + 1), big)
            for j in range(1, n):
                if edge in (WEST, EAST):
                    ii = h if edge == WEST else h + n
                    # centres on either side of the edge line, rows j-1 and j
                    a_lo = _normalize(C[:, ii - 1, h + j - 1] + C[:, ii, h + j - 1])
                    a_hi = _normalize(C[:, ii - 1, h + j] + C[:, ii, h + j])
                    corner = P[:, ii, h + j]
                else:
                    jj = h if edge == SOUTH else h + n
                    a_lo = _normalize(C[:, h + j - 1, jj - 1] + C[:, h + j - 1, jj])
                    a_hi = _normalize(C[:, h + j, jj - 1] + C[:, h + j, jj])
                    corner = P[:, h + j, jj]
                d1 = _gc_dist(a_lo, corner)
                d2 = _gc_dist(a_hi, corner)
                e[:, j] = d2 / (d1 + d2)
            out.append(e)
        return out

    def _cubed_to_latlon(self, C, me, mn):
        """a11, a12, a21, a22 of the cell-centre winds' transformation to
        longitude and latitude components (fv3core/grid/geometry.py:588-601):
        z = projections of the local grid directions ec1 (x, towards the east
        edge midpoint) and ec2 (y, towards the north edge midpoint) on the
        local east and north unit vectors, divided by sin_sg5."""
        _, _, east, north = lonlat_basis(C)
        ec1 = _tangent(C, me)
        ec2 = _tangent(C, mn)
        z11 = np.sum(ec1 * east, axis=-1)
        z12 = np.sum(ec1 * north, axis=-1)
        z21 = np.sum(ec2 * east, axis=-1)
        z22 = np.sum(ec2 * north, axis=-1)
        s5 = self.sin_sg5[:, : C.shape[1], : C.shape[2]]
        for name, val in (("a11", 0.5 * z22 / s5), ("a12", -0.5 * z12 / s5), ("a21", -0.5 * z21 / s5),
                          ("a22", 0.5 * z11 / s5)):
            out = np.zeros(self.shape2d)
            out[:, : C.shape[1], : C.shape[2]] = val
            setattr(self, name, out)

    # ------------------------------------------------------------------ helpers
    def wind_vectors(self):
        """Unit vectors along the D-grid edges: ex at u points (X, Y_INTERFACE),
        ey at v points (X_INTERFACE, Y), plus their midpoints."""
        P = self.corners
        mu = _normalize(P[:, :-1, :] + P[:, 1:, :])
        eu = _tangent(mu, P[:, 1:, :])
        mv = _normalize(P[:, :, :-1] + P[:, :, 1:])
        ev = _tangent(mv, P[:, :, 1:])
        return mu, eu, mv, ev


def lonlat_basis(p):
    """Local east and north unit vectors at unit position vectors p."""
    lon, lat = _lonlat(p)
    east = np.stack([-np.sin(lon), np.cos(lon), np.zeros_like(lon)], axis=-1)
    north = np.stack([-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)], axis=-1)
    return lon, lat, east, north
