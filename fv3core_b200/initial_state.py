"""Vertical coordinate and the Jablonowski-Williamson (2006) baroclinic-wave
initial state, in the form the acoustic substep consumes.

The reference takes this state from Fortran (``test_case: 13``); it is not in
the reference checkout, so it is written here from the published JW06
formulas.  Moisture follows the reference's ``fv_setup`` with nwat=6
(``fv3core/stencils/moist_cv.py:197-228``): four seeded tracers fill qvapor,
qliquid, qrain and qice, from which q_con, cappa and pkz are derived, and pt
is converted to the dynamics' virtual potential temperature
(``fv3core/stencils/fv_dynamics.py:32-34``).
"""
import numpy as np

from . import constants as C
from .grid import CubedSphereGrid, lonlat_basis
from .halo_map import apply_scalar_table, apply_vector_tables, scalar_table, vector_tables

P_REF = 1.0e5
CV_VAP = 3.0 * C.RVGAS
C_LIQ = 4.1855e3
C_ICE = 1972.0


def hybrid_coordinate(nz, ptop=300.0, eta_c=0.15):
    """Smooth hybrid sigma-pressure coordinate with ``nz`` layers.

    Interface pressures for a 1000 hPa surface are spaced by a blend of a
    uniform and a cosine profile (finer near the top and the surface); ``bk``
    is zero above eta_c and rises quadratically to 1 at the surface.
    Returns (ak, bk, ptop, ks) with ks the number of pure-pressure layers.
    """
    s = np.linspace(0.0, 1.0, nz + 1)
    f = 0.55 * s + 0.45 * 0.5 * (1.0 - np.cos(np.pi * s))
    p = ptop + (P_REF - ptop) * f
    eta = p / P_REF
    bk = np.where(eta > eta_c, ((eta - eta_c) / (1.0 - eta_c)) ** 2, 0.0)
    bk[-1] = 1.0
    ak = p - bk * P_REF
    ak[-1] = 0.0
    ak[0] = ptop
    ks = int(np.count_nonzero(bk == 0.0)) - 1
    return ak, bk, ptop, ks


# JW06 parameters
_ETA0, _ETAT, _U0, _T0, _GAMMA, _DT = 0.252, 0.2, 35.0, 288.0, 0.005, 4.8e5


def _jw_temperature(eta, lat):
    etav = (eta - _ETA0) * 0.5 * np.pi
    tbar = _T0 * eta ** (C.RDGAS * _GAMMA / C.GRAV)
    tbar = np.where(eta < _ETAT, tbar + _DT * (_ETAT - eta) ** 5, tbar)
    sl, cl = np.sin(lat), np.cos(lat)
    term1 = (-2.0 * sl**6 * (cl**2 + 1.0 / 3.0) + 10.0 / 63.0) * 2.0 * _U0 * np.cos(etav) ** 1.5
    term2 = (1.6 * cl**3 * (sl**2 + 2.0 / 3.0) - 0.25 * np.pi) * C.RADIUS * C.OMEGA
    return tbar + 0.75 * eta * np.pi * _U0 / C.RDGAS * np.sin(etav) * np.sqrt(np.cos(etav)) * (term1 + term2)


def _jw_surface_geopotential(lat):
    etav = (1.0 - _ETA0) * 0.5 * np.pi
    sl, cl = np.sin(lat), np.cos(lat)
    return _U0 * np.cos(etav) ** 1.5 * (
        (-2.0 * sl**6 * (cl**2 + 1.0 / 3.0) + 10.0 / 63.0) * _U0 * np.cos(etav) ** 1.5
        + (1.6 * cl**3 * (sl**2 + 2.0 / 3.0) - 0.25 * np.pi) * C.RADIUS * C.OMEGA
    )


def _jw_u(eta, lat):
    etav = (eta - _ETA0) * 0.5 * np.pi
    return _U0 * np.cos(etav) ** 1.5 * np.sin(2.0 * lat) ** 2


class AcousticState(dict):
    """Dict of numpy FP64 fields ``[6, n+2h+1, n+2h+1, nz+1]`` (2-D fields
    ``[6, n+2h+1, n+2h+1]``, 1-D ``[nz+1]``) plus scalars, named as in the
    reference's ``AcousticDynamics`` state namespace."""


def baroclinic_state(grid: CubedSphereGrid, nz, seed=0, noise=1.0e-3, ntracers=4):
    n, h = grid.n, grid.halo
    m = n + 2 * h + 1
    rng = np.random.default_rng(seed)
    ak, bk, ptop, ks = hybrid_coordinate(nz)
    shape3 = (6, m, m, nz + 1)
    st = AcousticState()
    # ---- pressure column at cell centres (surface pressure 1000 hPa everywhere)
    ps = P_REF
    pe_col = ak + bk * ps
    delp_col = np.diff(pe_col)
    pmid = delp_col / np.log(pe_col[1:] / pe_col[:-1])
    eta_mid = pmid / P_REF
    lat_a = grid.lat_a
    lat_b = grid.lat_b
    T = _jw_temperature(eta_mid[None, None, None, :], lat_a[..., None])
    # ---- tracers (qvapor, qliquid, qrain, qice) uniform in [0, 1e-2)
    q = rng.uniform(0.0, 1.0e-2, size=(ntracers, 6, m, m, nz))
    qv, ql, qr, qi = (q[i] if i < ntracers else np.zeros((6, m, m, nz)) for i in range(4))
    q_con = ql + qr + qi
    cvm = (1.0 - (qv + q_con)) * C.CV_AIR + qv * CV_VAP + (ql + qr) * C_LIQ + qi * C_ICE
    dp1 = C.ZVIR * qv
    cappa = C.RDGAS / (C.RDGAS + cvm / (1.0 + dp1))
    # seeded relative noise on temperature
    T = T * (1.0 + noise * rng.standard_normal(T.shape))
    Tv = T * (1.0 + dp1) * (1.0 - q_con)
    delz = -C.RDGAS * Tv / C.GRAV * np.log(pe_col[1:] / pe_col[:-1])
    delp = np.broadcast_to(delp_col, T.shape).copy()
    pkz = np.exp(cappa * np.log(C.RDG * delp * T * (1.0 + dp1) * (1.0 - q_con) / delz))
    pt = T * (1.0 + dp1) * (1.0 - q_con) / pkz

    def full(a3):
        out = np.zeros(shape3)
        out[..., : a3.shape[-1]] = a3
        return out

    for name, q_ in (("qvapor", qv), ("qliquid", ql), ("qrain", qr), ("qice", qi)):
        st[name] = full(q_)
    st["delp"] = full(delp)
    st["pt"] = full(pt)
    st["delz"] = full(delz)
    st["q_con"] = full(q_con)
    st["cappa"] = full(cappa)
    st["pkz"] = full(pkz)
    st["w"] = np.zeros(shape3)
    # ---- winds: zonal jet projected on the D-grid edges, seeded noise
    mu, eu, mv, ev = grid.wind_vectors()
    _, latu, eastu, _ = lonlat_basis(mu)
    _, latv, eastv, _ = lonlat_basis(mv)
    uz_u = _jw_u(eta_mid[None, None, None, :], latu[..., None])
    uz_v = _jw_u(eta_mid[None, None, None, :], latv[..., None])
    u = uz_u * np.sum(eastu * eu, axis=-1)[..., None]
    v = uz_v * np.sum(eastv * ev, axis=-1)[..., None]
    u = u * (1.0 + noise * rng.standard_normal(u.shape))
    v = v + noise * np.abs(uz_v) * rng.standard_normal(v.shape)
    uf = np.zeros(shape3)
    uf[:, : m - 1, :, :nz] = u
    vf = np.zeros(shape3)
    vf[:, :, : m - 1, :nz] = v
    st["u"], st["v"] = uf, vf
    # ---- surface geopotential and interface pressures
    phis = np.zeros((6, m, m))
    phis[:, : m - 1, : m - 1] = _jw_surface_geopotential(lat_a[:, : m - 1, : m - 1])
    st["phis"] = phis
    pe = np.broadcast_to(pe_col, shape3).copy()
    st["pe"] = pe
    st["peln"] = np.log(pe)
    st["pk"] = np.exp(C.KAPPA * st["peln"])
    for name in ("uc", "vc", "ua", "va", "omga", "mfxd", "mfyd", "cxd", "cyd", "diss_estd"):
        st[name] = np.zeros(shape3)
    st["wsd"] = np.zeros((6, m, m))
    st["ak"], st["bk"] = ak, bk
    ph1 = ak[:-1] + bk[:-1] * P_REF
    ph2 = ak[1:] + bk[1:] * P_REF
    pfull = np.zeros(nz + 1)
    pfull[:nz] = (ph2 - ph1) / np.log(ph2 / ph1)
    st["pfull"] = pfull
    st["ptop"] = float(ptop)
    st["ks"] = int(ks)
    # ---- make halos consistent with the neighbouring tiles
    tc = scalar_table(n, h, 1, 1, h)
    for name in ("delp", "pt", "delz", "q_con", "cappa", "pkz", "pe", "peln", "pk", "qvapor", "qliquid", "qrain",
                 "qice"):
        apply_scalar_table(st[name], tc)
    apply_scalar_table(st["phis"], tc)
    apply_vector_tables(st["u"], st["v"], vector_tables(n, h, (1, 0), (0, 1), h))
    return st


def resting_state(grid: CubedSphereGrid, nz, temperature=280.0):
    """A dry isothermal atmosphere at rest over a flat surface, in the layout
    of ``baroclinic_state``: every column is the same hydrostatic column
    (delz from the interface log-pressures, pkz from the layer's log-mean
    pressure), u = v = w = 0 and phis = 0.  Acoustic substeps must leave the
    winds at zero and delp unchanged."""
    st = baroclinic_state(grid, nz, seed=0, noise=0.0, ntracers=0)
    pe_col = st["pe"][0, 0, 0, :]
    dlnp = np.log(pe_col[1:] / pe_col[:-1])
    delp_col = np.diff(pe_col)
    cappa = C.RDGAS / (C.RDGAS + C.CV_AIR)
    delz = -C.RDGAS * temperature / C.GRAV * dlnp
    pkz = np.exp(cappa * np.log(delp_col / dlnp))
    cols = {"delz": delz, "pkz": pkz, "pt": temperature / pkz, "cappa": np.full(nz, cappa),
            "q_con": np.zeros(nz)}
    for name, col in cols.items():
        st[name][..., :nz] = col
    for name in ("u", "v", "w", "phis"):
        st[name][...] = 0.0
    return st


STEP_TRACERS = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr", "qsgs_tke", "qcld")


def step_state(grid: CubedSphereGrid, nz, seed=0, noise=1.0e-3, base=None):
    """The baroclinic-wave state in the form DynamicalCore.step_dynamics
    takes it: ``baroclinic_state`` with its four seeded water species, the
    other species and the cloud fraction at zero, pt back as temperature
    (the step's preamble converts it, fv_dynamics.py:32-34, whose inverse is
    applied here) and the surface pressure ps."""
    st = baroclinic_state(grid, nz, seed=seed, noise=noise)
    shape3 = st["delp"].shape
    for name in STEP_TRACERS:
        if name not in st:
            st[name] = np.zeros(shape3)
    dp1 = C.ZVIR * st["qvapor"]
    with np.errstate(all="ignore"):
        t = st["pt"] * st["pkz"] / ((1.0 + dp1) * (1.0 - st["q_con"]))
    st["pt"] = np.where(np.isfinite(t), t, 0.0)
    st["ps"] = np.array(st["pe"][..., nz], copy=True)
    return st
