"""Cubed-sphere halo exchange.

fv3gfs-util (the reference's halo code) is not part of the reference
checkout, so parity of the exchange is pinned by geometry: after an exchange
the halo of a smooth field must equal the field evaluated at the halo cells'
own positions, for scalars at cell centres and corners and for D- and C-grid
wind components.  The oracle's slab implementation and the package's gather
tables (used by the CUDA kernel) must also agree point for point.
"""
import numpy as np
import pytest

import cases
from fv3core_b200 import halo_map as hm
from fv3core_b200.grid import lonlat_basis
from oracle.halo import HaloExchange

N = 12
H = 3


def _smooth(p):
    return 1.0 + 0.3 * p[..., 0] - 0.7 * p[..., 1] + 0.2 * p[..., 2] + 0.1 * p[..., 0] * p[..., 2]


def _rotation_wind(p):
    axis = np.array([0.3, -0.2, 0.9])
    axis = axis / np.linalg.norm(axis)
    return 20.0 * np.cross(axis, p)


def _edge_masks(n, h, sx, sy):
    """Boolean [m, m] masks of the compute domain and of the edge halos
    (corner blocks excluded) for staggering (sx, sy)."""
    m = n + 2 * h + 1
    ci = np.zeros(m, bool)
    ci[h : h + n + (1 - sx)] = True
    cj = np.zeros(m, bool)
    cj[h : h + n + (1 - sy)] = True
    hi = np.zeros(m, bool)
    hi[h - 3 : h] = True
    hi[h + n + (1 - sx) : h + n + (1 - sx) + 3] = True
    hj = np.zeros(m, bool)
    hj[h - 3 : h] = True
    hj[h + n + (1 - sy) : h + n + (1 - sy) + 3] = True
    halo = (hi[:, None] & cj[None, :]) | (ci[:, None] & hj[None, :])
    return halo


def test_scalar_halo_matches_geometry():
    g = cases.grid_for(N)
    m = N + 2 * H + 1
    f = np.zeros((6, m, m, 2))
    exact = np.zeros((6, m, m, 2))
    c = g.centers
    val = _smooth(c)
    exact[:, : m - 1, : m - 1, :] = val[..., None]
    f[:, H : H + N, H : H + N, :] = exact[:, H : H + N, H : H + N, :]
    HaloExchange(N, H).scalar(f)
    mask = _edge_masks(N, H, 1, 1)
    err = np.abs(f - exact)[:, mask]
    assert err.max() < 1e-12


def test_corner_scalar_halo_matches_geometry():
    g = cases.grid_for(N)
    m = N + 2 * H + 1
    exact = np.repeat(_smooth(g.corners)[..., None], 2, axis=-1)
    f = np.zeros_like(exact)
    f[:, H : H + N + 1, H : H + N + 1] = exact[:, H : H + N + 1, H : H + N + 1]
    HaloExchange(N, H).scalar_corner(f)
    mask = _edge_masks(N, H, 0, 0)
    assert np.abs(f - exact)[:, mask].max() < 1e-12


def _dgrid_exact(g):
    mu, eu, mv, ev = g.wind_vectors()
    m = g.n + 2 * g.halo + 1
    u = np.zeros((6, m, m, 1))
    v = np.zeros((6, m, m, 1))
    u[:, : m - 1, :, 0] = np.sum(_rotation_wind(mu) * eu, axis=-1)
    v[:, :, : m - 1, 0] = np.sum(_rotation_wind(mv) * ev, axis=-1)
    return u, v


def test_dgrid_vector_halo_matches_geometry():
    g = cases.grid_for(N)
    ue, ve = _dgrid_exact(g)
    u = np.zeros_like(ue)
    v = np.zeros_like(ve)
    u[:, H : H + N, H : H + N + 1] = ue[:, H : H + N, H : H + N + 1]
    v[:, H : H + N + 1, H : H + N] = ve[:, H : H + N + 1, H : H + N]
    HaloExchange(N, H).vector_d(u, v)
    mu_ = _edge_masks(N, H, 1, 0)
    mv_ = _edge_masks(N, H, 0, 1)
    assert np.abs(u - ue)[:, mu_].max() < 1e-10
    assert np.abs(v - ve)[:, mv_].max() < 1e-10


def test_cgrid_vector_halo_matches_geometry():
    """uc on (X_INTERFACE, Y) is the wind component across the cell edge
    normal to x, i.e. along the line joining cell centres."""
    g = cases.grid_for(N)
    c = g.centers
    m = N + 2 * H + 1
    # direction between neighbouring centres, at the midpoint
    pu = c[:, :-1, :] + c[:, 1:, :]
    pu = pu / np.linalg.norm(pu, axis=-1, keepdims=True)
    du = c[:, 1:, :] - c[:, :-1, :]
    du = du - np.sum(du * pu, axis=-1, keepdims=True) * pu
    du = du / np.linalg.norm(du, axis=-1, keepdims=True)
    pv = c[:, :, :-1] + c[:, :, 1:]
    pv = pv / np.linalg.norm(pv, axis=-1, keepdims=True)
    dv = c[:, :, 1:] - c[:, :, :-1]
    dv = dv - np.sum(dv * pv, axis=-1, keepdims=True) * pv
    dv = dv / np.linalg.norm(dv, axis=-1, keepdims=True)
    uce = np.zeros((6, m, m, 1))
    vce = np.zeros((6, m, m, 1))
    uce[:, 1 : m - 1, : m - 1, 0] = np.sum(_rotation_wind(pu) * du, axis=-1)
    vce[:, : m - 1, 1 : m - 1, 0] = np.sum(_rotation_wind(pv) * dv, axis=-1)
    uc = np.zeros_like(uce)
    vc = np.zeros_like(vce)
    uc[:, H : H + N + 1, H : H + N] = uce[:, H : H + N + 1, H : H + N]
    vc[:, H : H + N, H : H + N + 1] = vce[:, H : H + N, H : H + N + 1]
    HaloExchange(N, H).vector_c(uc, vc)
    # exact values need both neighbouring centres on the sphere: skip the
    # outermost interface and the south/north (west/east) halo points on the
    # tile-corner lines, whose other centre lies in a corner block
    mu_ = _edge_masks(N, H, 0, 1)
    mu_[[0, -1], :] = False
    mu_[[H, H + N], :H] = False
    mu_[[H, H + N], H + N :] = False
    mv_ = _edge_masks(N, H, 1, 0)
    mv_[:, [0, -1]] = False
    mv_[:H, [H, H + N]] = False
    mv_[H + N :, [H, H + N]] = False
    assert np.abs(uc - uce)[:, mu_].max() < 1e-10
    assert np.abs(vc - vce)[:, mv_].max() < 1e-10


@pytest.mark.parametrize("stagger", [(1, 1), (0, 0)])
@pytest.mark.parametrize("n_halo", [3, 2])
def test_package_tables_agree_with_oracle_scalar(stagger, n_halo):
    rng = np.random.default_rng(3)
    m = N + 2 * H + 1
    f = rng.standard_normal((6, m, m, 2))
    a = f.copy()
    b = f.copy()
    HaloExchange(N, H)._exchange([a], [stagger], False, n_halo, 2)
    hm.apply_scalar_table(b, hm.scalar_table(N, H, stagger[0], stagger[1], n_halo))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["d", "c"])
def test_package_tables_agree_with_oracle_vector(kind):
    rng = np.random.default_rng(4)
    m = N + 2 * H + 1
    x = rng.standard_normal((6, m, m, 2))
    y = rng.standard_normal((6, m, m, 2))
    xa, ya, xb, yb = x.copy(), y.copy(), x.copy(), y.copy()
    ex = HaloExchange(N, H)
    if kind == "d":
        ex.vector_d(xa, ya)
        st = ((1, 0), (0, 1))
    else:
        ex.vector_c(xa, ya)
        st = ((0, 1), (1, 0))
    hm.apply_vector_tables(xb, yb, hm.vector_tables(N, H, st[0], st[1], H))
    assert np.array_equal(xa, xb) and np.array_equal(ya, yb)


def test_sync_vector_interfaces_matches_tables():
    rng = np.random.default_rng(5)
    m = N + 2 * H + 1
    u = rng.standard_normal((6, m, m, 2))
    v = rng.standard_normal((6, m, m, 2))
    ua, va, ub, vb = u.copy(), v.copy(), u.copy(), v.copy()
    HaloExchange(N, H).sync_vector_interfaces(ua, va)
    rows = hm.interface_sync_tables(N, H)
    src = (ub.copy(), vb.copy())
    dst = (ub, vb)
    for r in rows:
        dst[r[1]][r[0], r[2], r[3]] = r[8] * src[r[5]][r[4], r[6], r[7]]
    assert np.array_equal(ua, ub) and np.array_equal(va, vb)


def test_sync_vector_interfaces_geometry():
    """After the sync, the two tiles sharing an edge hold the same physical
    wind component on the shared edge line (up to orientation)."""
    g = cases.grid_for(N)
    ue, ve = _dgrid_exact(g)
    u, v = ue.copy(), ve.copy()
    HaloExchange(N, H).sync_vector_interfaces(u, v)
    assert np.abs(u - ue).max() < 1e-10 and np.abs(v - ve).max() < 1e-10


def test_a2b_corner_ratios_match_the_oracle_formula():
    """The grid's precomputed a2b_ord4 corner-extrapolation ratios equal the
    oracle's on-the-fly great-circle formula bit for bit."""
    from oracle.a2b_ord4 import great_circle_dist

    from fv3core_b200.grid import CubedSphereGrid

    n, h = 12, 3
    g = CubedSphereGrid(n, h)
    s, e = h, h + n - 1
    corners = ((s, s), (e + 1, s), (e + 1, e + 1), (s, e + 1))
    for t in range(6):
        for c, (i, j) in enumerate(corners):
            b1, b2 = g.bgrid1[t, i, j], g.bgrid2[t, i, j]
            for m, ((di1, dj1), (di2, dj2)) in enumerate(g.A2B_CORNER_OFFSETS[c]):
                x1 = great_circle_dist(g.agrid1[t, i + di1, j + dj1], g.agrid2[t, i + di1, j + dj1], b1, b2)
                x2 = great_circle_dist(g.agrid1[t, i + di2, j + dj2], g.agrid2[t, i + di2, j + dj2], b1, b2)
                assert x1 / (x2 - x1) == g.a2b_extrap[t, c, m]
