"""Deterministic test cases shared by the golden-fixture generator (which runs
the reference here) and the parity tests (which run the oracle and the CUDA
path, on any machine).

Every case is built from the package's grid and baroclinic-wave generators
plus seeded perturbations, so only outputs need to be stored as fixtures.
Arrays are numpy FP64 in the reference's index order: 3-D fields
``[6, n+2h+1, n+2h+1, nz+1]``, 2-D ``[6, n+2h+1, n+2h+1]``.
"""
import functools

import numpy as np

from fv3core_b200 import constants as C
from fv3core_b200.grid import CubedSphereGrid
from fv3core_b200.initial_state import baroclinic_state

HALO = 3


# Face lattice of the cases' grid: the package's equiangular default, or
# "equidistant" (the reference's grid_type 0) for the fixtures made on the
# reference's own grid
LATTICE = "equiangular"


@functools.lru_cache(maxsize=8)
def _grid(n, lattice):
    return CubedSphereGrid(n, HALO, lattice=lattice)


def grid_for(n):
    return _grid(n, LATTICE)


def base_state(n, nz, seed):
    return baroclinic_state(grid_for(n), nz, seed=seed)


def heights(st, nz):
    """Interface heights (m) from delz and the surface height, as the
    reference's ``set_gz`` (dyn_core.py:80-85) builds them."""
    zs = st["phis"] / C.GRAV
    gz = np.zeros_like(st["delz"])
    gz[..., nz] = zs
    for k in range(nz - 1, -1, -1):
        gz[..., k] = gz[..., k + 1] - st["delz"][..., k]
    return gz


def riem_solver_c_case(n=12, nz=16, seed=11):
    st = base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    gz = heights(st, nz)
    case = {
        "dt2": 18.75,
        "ptop": st["ptop"],
        "p_fac": 0.05,
        "cappa": st["cappa"].copy(),
        "hs": st["phis"].copy(),
        "ws": 0.05 * rng.standard_normal(shp[:3]),
        "ptc": st["pt"] * (1.0 + 1e-3 * rng.standard_normal(shp)),
        "q_con": st["q_con"].copy(),
        "delpc": st["delp"] * (1.0 + 1e-3 * rng.standard_normal(shp)),
        "gz": gz * (1.0 + 1e-5 * rng.standard_normal(shp)),
        "pef": np.zeros(shp),
        "w3": 0.1 * rng.standard_normal(shp),
    }
    return case


CASES = {
    "riem_solver_c": riem_solver_c_case,
}


def metric_namespace(n, tile):
    """One tile's metric arrays as attributes (oracle input)."""
    import types

    g = grid_for(n)
    ns = types.SimpleNamespace()
    for name, val in vars(g).items():
        if isinstance(val, np.ndarray) and val.ndim == 3 and val.shape[0] == 6:
            setattr(ns, name, val[tile])
    for name in ("edge_w", "edge_e", "edge_s", "edge_n"):
        setattr(ns, name, getattr(g, name)[tile])
    ns.da_min, ns.da_min_c = g.da_min, g.da_min_c
    return ns


def c_sw_case(n=12, nz=6, seed=21):
    st = base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    r = lambda scale: scale * rng.standard_normal(shp)
    case = {
        "dt2": 18.75,
        "delp": st["delp"].copy(),
        "pt": st["pt"].copy(),
        "u": st["u"].copy(),
        "v": st["v"].copy(),
        "w": r(0.2),
        "uc": r(5.0),
        "vc": r(5.0),
        "ua": r(5.0),
        "va": r(5.0),
        "ut": r(5.0),
        "vt": r(5.0),
        "divgd": r(1e-5),
        "omga": r(0.1),
    }
    return case


CASES["c_sw"] = c_sw_case


# D-grid shallow-water namelist of the baroclinic-wave configuration
# (examples/wrapped/config/baroclinic.yml in the reference)
DSW_CONFIG = dict(
    dddmp=0.5, d2_bg=0.0, d2_bg_k1=0.2, d2_bg_k2=0.1, d4_bg=0.15, ke_bg=0.0, nord=3, n_sponge=48,
    grid_type=0, d_ext=0.0, hord_dp=6, hord_tm=6, hord_mt=6, hord_vt=6, do_f3d=False, do_skeb=False,
    d_con=1.0, vtdm4=0.06, inline_q=False, convert_ke=False, do_vort_damp=True, hydrostatic=False,
)


def d_sw_case(n=12, nz=8, seed=31):
    st = base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    r = lambda scale: scale * rng.standard_normal(shp)
    gz = heights(st, nz)
    case = {
        "dt": 37.5,
        "delpc": st["delp"] * (1.0 + 1e-3 * rng.standard_normal(shp)),
        "delp": st["delp"].copy(),
        "ptc": st["pt"] * (1.0 + 1e-3 * rng.standard_normal(shp)),
        "pt": st["pt"].copy(),
        "u": st["u"].copy(),
        "v": st["v"].copy(),
        "w": r(0.2),
        "uc": st["u"] * 0.9 + r(1.0),
        "vc": st["v"] * 0.9 + r(1.0),
        "ua": r(10.0),
        "va": r(10.0),
        "divgd": r(1e-5),
        "mfx": r(1e3),
        "mfy": r(1e3),
        "cx": r(0.05),
        "cy": r(0.05),
        "crx": r(0.05),
        "cry": r(0.05),
        "xfx": r(1e3),
        "yfx": r(1e3),
        "q_con": st["q_con"].copy(),
        "zh": gz,
        "heat_source": r(1e-3),
        "diss_est": r(1e-3),
    }
    return case


CASES["d_sw"] = d_sw_case


# Acoustic substep loop (AcousticDynamics) of the baroclinic configuration:
# acoustic namelist of examples/wrapped/config/baroclinic.yml in the reference,
# with n_split reduced so the six-tile reference run stays short.
ACOUSTIC_CONFIG = dict(
    tau=10.0, k_split=1, n_split=2, m_split=0, delt_max=0.002, rf_cutoff=3000.0, rf_fast=True,
    breed_vortex_inline=False, use_old_omega=True,
)
RIEMANN_CONFIG = dict(p_fac=0.05, a_imp=1.0, use_logp=False, beta=0.0)

ACOUSTIC_STATE = ["u", "v", "w", "delz", "delp", "pt", "pe", "pk", "phis", "wsd", "omga", "ua", "va", "uc",
                  "vc", "mfxd", "mfyd", "cxd", "cyd", "pkz", "peln", "q_con", "diss_estd", "cappa"]


def acoustics_case(n=12, nz=8, seed=41, n_split=2):
    st = base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    case = {name: np.array(st[name], copy=True) for name in ACOUSTIC_STATE if name in st}
    case["w"] = 0.1 * rng.standard_normal(shp)
    case["wsd"] = 0.01 * rng.standard_normal(shp[:3])
    for name in ("omga", "ua", "va", "uc", "vc", "mfxd", "mfyd", "cxd", "cyd", "diss_estd"):
        case[name] = np.zeros(shp)
    case.update(
        ak=np.asarray(st["ak"], dtype=np.float64), bk=np.asarray(st["bk"], dtype=np.float64),
        pfull=np.asarray(st["pfull"], dtype=np.float64), ptop=st["ptop"], ks=st["ks"],
        mdt=37.5 * n_split, n_map=1, akap=C.KAPPA, n_split=n_split,
    )
    return case


CASES["acoustics"] = acoustics_case


def smooth_acoustics_case(n=48, nz=79, n_split=6):
    """The baroclinic-wave state without seeded noise and without tracers
    (dry), w and the surface w at zero: a state smooth at the grid scale."""
    st = baroclinic_state(grid_for(n), nz, seed=0, noise=0.0, ntracers=0)
    shp = st["delp"].shape
    case = {name: np.array(st[name], copy=True) for name in ACOUSTIC_STATE if name in st}
    case["w"] = np.zeros(shp)
    case["wsd"] = np.zeros(shp[:3])
    for name in ("omga", "ua", "va", "uc", "vc", "mfxd", "mfyd", "cxd", "cyd", "diss_estd"):
        case[name] = np.zeros(shp)
    case.update(
        ak=np.asarray(st["ak"], dtype=np.float64), bk=np.asarray(st["bk"], dtype=np.float64),
        pfull=np.asarray(st["pfull"], dtype=np.float64), ptop=st["ptop"], ks=st["ks"],
        mdt=37.5 * n_split, n_map=1, akap=C.KAPPA, n_split=n_split,
    )
    return case
# the parity case of the plain FP64 method: C12 L79, one acoustic substep of
# dt_acoustic = 225 / 6 s (n_split = 1, mdt = 37.5 s)
CASES["acoustics_c12_l79"] = acoustics_case
CASES["acoustics_c12_l79_ed"] = acoustics_case


def resting_case(n=12, nz=8, n_split=2):
    """An acoustics case on a dry isothermal atmosphere at rest over a flat
    surface (identical hydrostatic columns, zero winds)."""
    from fv3core_b200.initial_state import resting_state

    st = resting_state(grid_for(n), nz)
    shp = st["delp"].shape
    case = {name: np.array(st[name], copy=True) for name in ACOUSTIC_STATE if name in st}
    case["wsd"] = np.zeros(shp[:3])
    for name in ("omga", "ua", "va", "uc", "vc", "mfxd", "mfyd", "cxd", "cyd", "diss_estd"):
        case[name] = np.zeros(shp)
    case.update(
        ak=np.asarray(st["ak"], dtype=np.float64), bk=np.asarray(st["bk"], dtype=np.float64),
        pfull=np.asarray(st["pfull"], dtype=np.float64), ptop=st["ptop"], ks=st["ks"],
        mdt=37.5 * n_split, n_map=1, akap=C.KAPPA, n_split=n_split,
    )
    return case


def tracer_case(n=12, nz=8, seed=61, ntracers=4, courant=0.6):
    """Inputs of TracerAdvection after an acoustic loop: four tracers uniform
    in [0, 1e-2), the pressure thickness dp1 of the baroclinic-wave state,
    and accumulated Courant numbers and mass fluxes of a smooth flow (the
    state's D-grid winds averaged to the C-grid interfaces, scaled to peak
    Courant number ``courant``) with seeded 1e-3 relative noise."""
    st = base_state(n, nz, seed)
    g = grid_for(n)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    u, v, dp = st["u"], st["v"], st["delp"]

    def sh(a, di, dj):
        out = np.zeros_like(a)
        m = a.shape[1]
        out[:, max(0, -di):m - max(0, di), max(0, -dj):m - max(0, dj)] = \
            a[:, max(0, di):m - max(0, -di), max(0, dj):m - max(0, -dj)]
        return out

    # x-interface (i - 1/2, j) and y-interface (i, j - 1/2) winds
    ux = 0.25 * (sh(u, -1, 0) + u + sh(u, -1, 1) + sh(u, 0, 1))
    vy = 0.25 * (sh(v, 0, -1) + v + sh(v, 1, -1) + sh(v, 1, 0))
    scale = courant / max(np.abs(ux).max(), np.abs(vy).max())
    cx = scale * ux * (1.0 + 1e-3 * rng.standard_normal(shp))
    cy = scale * vy * (1.0 + 1e-3 * rng.standard_normal(shp))
    dxa, dya, dx, dy = (getattr(g, k)[:, :, :, None] for k in ("dxa", "dya", "dx", "dy"))
    mfx = cx * 0.5 * (sh(dxa, -1, 0) + dxa) * dy * 0.5 * (sh(dp, -1, 0) + dp)
    mfy = cy * 0.5 * (sh(dya, 0, -1) + dya) * dx * 0.5 * (sh(dp, 0, -1) + dp)
    tracers = rng.uniform(0.0, 1.0e-2, size=(ntracers,) + shp)
    tracers[..., nz] = 0.0
    return {"tracers": tracers, "dp1": dp.copy(), "mfxd": mfx, "mfyd": mfy, "cxd": cx, "cyd": cy,
            "mdt": 225.0}


CASES["tracer_advection"] = tracer_case


WATER_NAMES = ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "qcld")


def fv_step_case(n=12, nz=8, seed=71):
    """Inputs of the step preamble and epilogue: the baroclinic-wave state
    with seven water species, uniform in [0, 1e-3), of which a seeded 20 %
    of the points are made negative (down to -2e-4) so that the negative
    tracer fixes act; the bottom level of qvapor stays non-negative (the
    reference's borrowing from below reads a temporary it only writes on the
    bottom level)."""
    st = base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    case = {k: np.array(st[k], copy=True) for k in ("delp", "delz", "pt", "u", "v", "peln")}
    for name in WATER_NAMES:
        q = rng.uniform(0.0, 1.0e-3, shp)
        neg = rng.random(shp) < 0.2
        q = np.where(neg, -rng.uniform(0.0, 2.0e-4, shp), q)
        if name == "qvapor":
            q[..., nz - 1] = np.abs(q[..., nz - 1])
        q[..., nz] = 0.0
        case[name] = q
    case["w"] = 0.1 * rng.standard_normal(shp)
    for name in ("q_con", "cvm", "pkz", "cappa", "dp1", "omga", "ua", "va"):
        case[name] = np.zeros(shp)
    return case


CASES["fv_step"] = fv_step_case


# Tracers of the remapping step, in the reference's order (utils.tracer_variables,
# the first NQ = 8 are remapped by MapNTracer); qcld is remapped only by the
# saturation adjustment, which this case leaves out.
REMAP_TRACERS = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr", "qsgs_tke")
# Remapping namelist of the baroclinic-wave configuration
# (examples/wrapped/config/baroclinic.yml in the reference), without the
# saturation adjustment.
REMAP_CONFIG = dict(fill=True, kord_tm=-9, kord_tr=9, kord_wz=9, kord_mt=9, do_sat_adj=False)
# fast saturation adjustment namelist (baroclinic.yml values, the reference's
# Namelist defaults for the rest)
SAT_ADJUST_CONFIG = dict(
    hydrostatic=False, rad_snow=True, rad_rain=True, rad_graupel=True, tintqs=False, sat_adj0=0.9, ql_gen=1.0e-3,
    qs_mlt=1.0e-6, ql0_max=2.0e-3, t_sub=184.0, qi_gen=1.82e-6, qi_lim=1.0, qi0_max=1.0e-4, dw_ocean=0.1,
    dw_land=0.15, icloud_f=0, cld_min=0.05, tau_i2s=1000.0, tau_v2l=90.0, tau_r2g=900.0, tau_l2r=900.0,
    tau_l2v=300.0, tau_imlt=600.0, tau_smlt=900.0,
)
REMAP_STATE = ("pt", "delp", "delz", "peln", "u", "v", "w", "ua", "va", "cappa", "q_con", "pkz", "pk", "pe",
               "ps", "te0_2d", "wsd")


def remap_case(n=12, nz=8, seed=81, kord=(-9, 9, 9, 9), sat_adj=False):
    """Inputs of LagrangianToEulerian: the baroclinic-wave state whose layer
    thicknesses are perturbed by a seeded factor in [0.7, 1.3] at every
    point (halo included), so that the Lagrangian surfaces pe (ptop plus the
    running sum of delp) leave the Eulerian ak + bk ps levels, some target
    layers spanning three source layers; peln, pk and
    the hydrostatic delz follow from pe.  Eight tracers uniform in
    [0, 1e-3), of which a seeded 3 % of the points are negative (down to
    -1e-4) so that the negative-value filling acts; w and the bottom w
    boundary wsd are seeded noise.  ``kord`` gives (kord_tm, kord_tr,
    kord_wz, kord_mt); ``sat_adj`` turns on the fast saturation adjustment
    (cloud fraction qcld then seeded in [0, 1))."""
    st = base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 1000)
    shp = st["delp"].shape
    ptop = st["ptop"]
    delp = st["delp"][..., :nz] * rng.uniform(0.7, 1.3, shp[:3] + (nz,))
    pe = np.empty(shp)
    pe[..., 0] = ptop
    pe[..., 1:] = ptop + np.cumsum(delp, axis=-1)
    pe_col = st["pe"][0, 0, 0, :]
    ratio = np.log(pe[..., 1:] / pe[..., :-1]) / np.log(pe_col[1:] / pe_col[:-1])
    case = {k: np.array(st[k], copy=True) for k in ("pt", "u", "v", "cappa", "q_con", "pkz", "phis")}
    case["delp"] = np.zeros(shp)
    case["delp"][..., :nz] = delp
    case["delz"] = np.zeros(shp)
    case["delz"][..., :nz] = st["delz"][..., :nz] * ratio
    case["pe"] = pe
    case["peln"] = np.log(pe)
    case["pk"] = np.exp(C.KAPPA * case["peln"])
    case["w"] = 0.1 * rng.standard_normal(shp)
    case["wsd"] = 0.05 * rng.standard_normal(shp[:3])
    case["ps"] = np.zeros(shp[:3])
    case["te0_2d"] = np.zeros(shp[:3])
    case["ua"] = np.zeros(shp)
    case["va"] = np.zeros(shp)
    for name in REMAP_TRACERS:
        q = rng.uniform(0.0, 1.0e-3, shp)
        neg = rng.random(shp) < 0.03
        q = np.where(neg, -rng.uniform(0.0, 1.0e-4, shp), q)
        q[..., nz] = 0.0
        case[name] = q
    case["qcld"] = rng.uniform(0.0, 1.0, shp) if sat_adj else np.zeros(shp)
    case["dp1"] = np.zeros(shp)
    case["omga"] = np.zeros(shp)
    case["ak"], case["bk"], case["pfull"] = st["ak"], st["bk"], st["pfull"]
    case["ptop"] = ptop
    case["mdt"] = 225.0
    case["kord"] = np.array(kord)
    case["do_sat_adj"] = np.array(bool(sat_adj))
    return case


def remap_config(case):
    """The remapping namelist of a remap case (its kord values)."""
    kord_tm, kord_tr, kord_wz, kord_mt = (int(x) for x in case["kord"])
    return dict(REMAP_CONFIG, kord_tm=kord_tm, kord_tr=kord_tr, kord_wz=kord_wz, kord_mt=kord_mt,
                do_sat_adj=bool(case.get("do_sat_adj", False)))


CASES["remap"] = remap_case
# the profile's other limiters: kord 10 (ext5 / ext6 tests) and kord 8
CASES["remap_kord10"] = functools.partial(remap_case, kord=(-10, 10, 10, 10))
CASES["remap_kord8"] = functools.partial(remap_case, kord=(-8, 8, 8, 8))
# the baroclinic namelist's remapping with the fast saturation adjustment
CASES["remap_satadj"] = functools.partial(remap_case, sat_adj=True)


# the water species and tracers of DynamicalCore's state: the eight it
# advects and remaps (NQ = 8) and qcld
STEP_TRACERS = REMAP_TRACERS + ("qcld",)


def step_case(n=12, nz=12, seed=101, n_split=2, sat_adj=False):
    """Inputs of DynamicalCore.step_dynamics (one k_split step of
    dt_atmos = 225 s, n_split acoustic substeps): the acoustics case's
    baroclinic-wave state with its potential temperature turned back into a
    temperature (pt pkz, step_dynamics converts it in its preamble), water
    vapour uniform in [1e-4, 1e-2), the other species in [0, 1e-5) with a
    seeded 2 % of negative points (down to -1e-6), cloud fraction in
    [0, 0.5); ``sat_adj`` turns on the remapping's fast saturation
    adjustment."""
    case = acoustics_case(n, nz, seed, n_split)
    rng = np.random.default_rng(seed + 2000)
    shp = case["delp"].shape
    case["pt"] = case["pt"] * case["pkz"]
    for name in STEP_TRACERS:
        if name == "qvapor":
            q = rng.uniform(1.0e-4, 1.0e-2, shp)
        elif name == "qcld":
            q = rng.uniform(0.0, 0.5, shp)
        else:
            q = rng.uniform(0.0, 1.0e-5, shp)
            neg = rng.random(shp) < 0.02
            q = np.where(neg, -rng.uniform(0.0, 1.0e-6, shp), q)
        q[..., nz] = 0.0
        case[name] = q
    case["ps"] = np.array(case["pe"][..., nz], copy=True)
    case["mdt"] = 225.0
    case["dt_atmos"] = 225.0
    case["do_sat_adj"] = np.array(bool(sat_adj))
    return case


CASES["step"] = step_case
CASES["step_satadj"] = functools.partial(step_case, sat_adj=True)


def dycore_namelist(n, nz, n_split, sat_adj=False):
    """DynamicalCoreConfig values of the baroclinic-wave configuration
    (examples/wrapped/config/baroclinic.yml in the reference) on a C``n``
    L``nz`` grid, without the saturation adjustment."""
    nl = dict(DSW_CONFIG)
    nl.update({k: v for k, v in ACOUSTIC_CONFIG.items()})
    nl.update(RIEMANN_CONFIG)
    nl.update({k: v for k, v in REMAP_CONFIG.items()})
    nl.update(SAT_ADJUST_CONFIG)
    nl.update(dt_atmos=225, consv_te=False, hord_tr=8, z_tracer=True, nwat=6, npx=n + 1, npy=n + 1, npz=nz,
              ntiles=6, do_qa=True, n_split=n_split, moist_phys=True, c2l_ord=4, p_ref=1e5, nf_omega=1,
              do_sat_adj=bool(sat_adj))
    return nl


def gnomonic_case(n=12, nz=1, seed=0):
    """The reference's grid_type 0 face takes no inputs but its size."""
    return {}


CASES["gnomonic_ed_c12"] = gnomonic_case
CASES["gnomonic_ed_c48"] = gnomonic_case
