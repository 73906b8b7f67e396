"""Generate golden fixtures by running the reference's own stencil classes.

Run on a machine that holds the reference checkout::

    FV3CORE_REFERENCE=<checkout> python tests/golden/make_golden.py [case ...]

For each case in ``cases.py`` the inputs are rebuilt deterministically, the
reference class runs tile by tile (or, for the full substep, six tiles in
lock step with a threaded halo exchange), and the outputs are stored in
``tests/golden/<case>.npz`` restricted to the points the reference defines.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import cases  # noqa: E402
import reference_runner as rr  # noqa: E402


def run_riem_solver_c(case, n, nz):
    from fv3core.stencils.riem_solver_c import RiemannSolverC

    grid = cases.grid_for(n)
    out = {"pef": np.zeros_like(case["pef"]), "gz": np.zeros_like(case["gz"])}
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        rs = RiemannSolverC(tr.stencil_factory, p_fac=case["p_fac"])
        S = rr.storage
        pef = S(case["pef"][t])
        gz = S(case["gz"][t])
        rs(
            case["dt2"],
            S(case["cappa"][t]),
            case["ptop"],
            S(case["hs"][t], origin=(3, 3)),
            S(case["ws"][t], origin=(3, 3)),
            S(case["ptc"][t]),
            S(case["q_con"][t]),
            S(case["delpc"][t]),
            gz,
            pef,
            S(case["w3"][t]),
        )
        out["pef"][t] = pef
        out["gz"][t] = gz
    h = 3
    sl = (slice(None), slice(h - 1, h + n + 1), slice(h - 1, h + n + 1), slice(0, nz + 1))
    return {k: v[sl] for k, v in out.items()}, {"region": "is-1:ie+2, js-1:je+2, 0:nz+1"}


def run_c_sw(case, n, nz):
    from fv3core.stencils.c_sw import CGridShallowWaterDynamics

    grid = cases.grid_for(n)
    names = ["delp", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "ut", "vt", "divgd", "omga"]
    out = {k: np.zeros_like(case["delp"]) for k in names + ["delpc", "ptc"]}
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        csw = CGridShallowWaterDynamics(tr.stencil_factory, tr.grid_data, False, 0, 3)
        st = {k: rr.storage(case[k][t]) for k in names}
        delpc, ptc = csw(*[st[k] for k in names], case["dt2"])
        for k in names:
            out[k][t] = st[k]
        out["delpc"][t] = delpc
        out["ptc"][t] = ptc
    return out, {"region": "full storage"}


DSW_ARGS = ["delpc", "delp", "ptc", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "divgd", "mfx", "mfy",
            "cx", "cy", "crx", "cry", "xfx", "yfx", "q_con", "zh", "heat_source", "diss_est"]


def run_d_sw(case, n, nz):
    from fv3core._config import DGridShallowWaterLagrangianDynamicsConfig
    from fv3core.stencils import d_sw

    grid = cases.grid_for(n)
    cfg = DGridShallowWaterLagrangianDynamicsConfig(**cases.DSW_CONFIG)
    out = {k: np.zeros_like(case["delp"]) for k in DSW_ARGS}
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        col = d_sw.get_column_namelist(cfg, nz)
        dsw = d_sw.DGridShallowWaterLagrangianDynamics(
            tr.stencil_factory, tr.grid_data, tr.damping_coefficients, col, False, False, cfg
        )
        st = {k: rr.storage(case[k][t]) for k in DSW_ARGS}
        dsw(*[st[k] for k in DSW_ARGS], case["dt"])
        for k in DSW_ARGS:
            out[k][t] = st[k]
    return out, {"region": "full storage"}


ACOUSTIC_DIMS = {
    "u": ("x", "y_interface", "z"), "v": ("x_interface", "y", "z"), "uc": ("x_interface", "y", "z"),
    "vc": ("x", "y_interface", "z"), "w": ("x", "y", "z"), "delp": ("x", "y", "z"), "pt": ("x", "y", "z"),
    "q_con": ("x", "y", "z"), "cappa": ("x", "y", "z"),
}


def run_acoustics(case, n, nz):
    """Six AcousticDynamics instances (one per tile) stepping in lock step on
    threads, their halo updates going through ``ThreadComm``."""
    import threading
    import types

    from fv3core._config import (AcousticDynamicsConfig, DGridShallowWaterLagrangianDynamicsConfig,
                                 RiemannConfig)
    from fv3core.stencils.dyn_core import AcousticDynamics
    from fv3core.utils.grid import quantity_wrap

    grid = cases.grid_for(n)
    cfg = AcousticDynamicsConfig(
        **{**cases.ACOUSTIC_CONFIG, "n_split": int(case["n_split"])},
        riemann=RiemannConfig(**cases.RIEMANN_CONFIG),
        d_grid_shallow_water=DGridShallowWaterLagrangianDynamicsConfig(**cases.DSW_CONFIG),
    )
    exchange = rr._Exchange()
    S = rr.storage
    runs = []
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        tr.activate()
        comm = rr.ThreadComm(t, n, 3, exchange)
        ak, bk, pfull = (S(case[k], origin=(0,)) for k in ("ak", "bk", "pfull"))
        phis = S(case["phis"][t], origin=(0, 0))
        ad = AcousticDynamics(comm, tr.stencil_factory, tr.grid_data, tr.damping_coefficients, 0, False, False,
                              cfg, ak, bk, pfull, phis)
        state = types.SimpleNamespace()
        for name in cases.ACOUSTIC_STATE:
            arr = case[name][t]
            setattr(state, name, S(arr, origin=(3, 3) if arr.ndim == 2 else (3, 3, 0)))
        for name, dims in ACOUSTIC_DIMS.items():
            setattr(state, name + "_quantity", quantity_wrap(getattr(state, name), dims, tr.grid_indexing))
        state.ak, state.bk, state.pfull = ak, bk, pfull
        for name in ("mdt", "n_map", "akap", "ptop", "ks"):
            setattr(state, name, case[name])
        runs.append((ad, state))
    errors = []

    def work(ad, state):
        try:
            ad(state)
        except BaseException as exc:  # surfaced after join
            errors.append(exc)
            raise

    threads = [threading.Thread(target=work, args=r) for r in runs]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    out = {name: np.stack([np.asarray(getattr(st, name)) for _, st in runs]) for name in cases.ACOUSTIC_STATE}
    for name in ("zh", "gz", "pkc", "pk3", "heat_source", "delpc", "ptc", "divgd"):
        out["tmp_" + name] = np.stack([np.asarray(getattr(st, name)) for _, st in runs])
    return out, {"region": "full storage"}


# fields of the C12 L79 fixture: the prognostic fields and the edge
# pressures, on the compute domain (the full storages of 24 fields at L79
# would make a 40 MB fixture)
L79_FIELDS = {"u": (0, 1, 0), "v": (1, 0, 0), "w": (0, 0, 0), "delp": (0, 0, 0), "pt": (0, 0, 0),
              "delz": (0, 0, 0), "q_con": (0, 0, 0), "pe": (0, 0, 1), "pk": (0, 0, 1), "peln": (0, 0, 1),
              "pkz": (0, 0, 0)}


def run_acoustics_compute(case, n, nz):
    out, _ = run_acoustics(case, n, nz)
    h = 3
    res = {}
    for name, (di, dj, dk) in L79_FIELDS.items():
        res[name] = out[name][:, h:h + n + di, h:h + n + dj, :nz + dk]
    return res, {"region": "compute domain (+1 on staggered axes)"}


TRACER_NAMES = ("qvapor", "qliquid", "qrain", "qsnow")


def run_tracer_advection(case, n, nz):
    """Six TracerAdvection instances (one per tile, hord_tr = 8 transport)
    stepping in lock step on threads, their tracer halo updates going
    through ``ThreadComm``, as DynamicalCore._dyn calls them after the
    acoustic loop (fv_dynamics.py:301-309, 544-557)."""
    import threading

    from fv3core.stencils.fvtp2d import FiniteVolumeTransport
    from fv3core.stencils.tracer_2d_1l import TracerAdvection
    from fv3core.utils.grid import quantity_wrap

    grid = cases.grid_for(n)
    exchange = rr._Exchange()
    S = rr.storage
    ntr = case["tracers"].shape[0]
    dims = ("x", "y", "z")
    runs = []
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        tr.activate()
        tr.add_tracer_grid()
        comm = rr.ThreadComm(t, n, 3, exchange)
        transport = FiniteVolumeTransport(tr.stencil_factory, tr.grid_data, tr.damping_coefficients, 0, hord=8)
        adv = TracerAdvection(tr.stencil_factory, transport, comm, ntr)
        tracers = {TRACER_NAMES[q]: quantity_wrap(S(case["tracers"][q, t]), dims, tr.grid_indexing)
                   for q in range(ntr)}
        args = {k: S(case[k][t]) for k in ("dp1", "mfxd", "mfyd", "cxd", "cyd")}
        runs.append((adv, tracers, args))
    errors = []

    def work(adv, tracers, args):
        try:
            adv(tracers, args["dp1"], args["mfxd"], args["mfyd"], args["cxd"], args["cyd"], case["mdt"])
        except BaseException as exc:  # surfaced after join
            errors.append(exc)
            raise

    threads = [threading.Thread(target=work, args=r) for r in runs]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    out = {"tracers": np.stack([np.stack([np.asarray(r[1][TRACER_NAMES[q]].storage) for r in runs])
                                for q in range(ntr)])}
    for k in ("dp1", "mfxd", "mfyd", "cxd", "cyd"):
        out[k] = np.stack([np.asarray(r[2][k]) for r in runs])
    return out, {"region": "full storage"}


FV_STEP_FIELDS = cases.WATER_NAMES + ("q_con", "cvm", "pkz", "pt", "cappa", "delp", "delz", "dp1", "w", "omga",
                                      "u", "v", "ua", "va", "peln")


def run_fv_step(case, n, nz):
    """The step preamble, post_remap and wrapup of DynamicalCore
    (fv_dynamics.py:54-169) on six tiles in lock step on threads, with the
    stencils built as DynamicalCore.__init__ builds them (fv_dynamics.py
    320-392); the state after each phase is stored (prefixes pre_, post_,
    wrap_)."""
    import threading
    import types

    from fv3core.stencils import fv_dynamics as fvd
    from fv3core.stencils import moist_cv
    from fv3core.stencils.c2l_ord import CubedToLatLon
    from fv3core.stencils.del2cubed import HyperdiffusionDamping
    from fv3core.stencils.neg_adj3 import AdjustNegativeTracerMixingRatio
    from fv3core.utils.grid import quantity_wrap

    grid = cases.grid_for(n)
    exchange = rr._Exchange()
    S = rr.storage
    config = types.SimpleNamespace(hydrostatic=False, rf_fast=True, tau=10.0, adiabatic=False, kord_tm=-9,
                                   nf_omega=1, nwat=6, moist_phys=True)
    runs = []
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        tr.activate()
        tr.add_tracer_grid()
        comm = rr.ThreadComm(t, n, 3, exchange)
        sf, gi = tr.stencil_factory, tr.grid_indexing
        fv_setup = sf.from_origin_domain(moist_cv.fv_setup, externals={"nwat": 6, "moist_phys": True},
                                         origin=gi.origin_compute(), domain=gi.domain_compute())
        pt_adjust = sf.from_origin_domain(fvd.pt_adjust, origin=gi.origin_compute(), domain=gi.domain_compute())
        set_omega = sf.from_origin_domain(fvd.set_omega, origin=gi.origin_compute(), domain=gi.domain_compute())
        hyper = HyperdiffusionDamping(sf, tr.damping_coefficients, tr.grid_data.rarea, config.nf_omega)
        c2l = CubedToLatLon(sf, tr.grid_data, order=4)
        adjust = AdjustNegativeTracerMixingRatio(sf, False, False)
        spec = gi.get_quantity_halo_spec(gi.domain_full(add=(1, 1, 1)), gi.origin_compute(),
                                         dims=["x", "y", "z"], n_halo=3)
        omega_updater = comm.get_scalar_halo_updater([spec])
        st = types.SimpleNamespace(**{k: S(case[k][t]) for k in FV_STEP_FIELDS})
        st.consv_te = 0.0
        st.do_adiabatic_init = False
        st.omga_quantity = quantity_wrap(st.omga, ("x", "y", "z"), gi)
        st.u_quantity = quantity_wrap(st.u, ("x", "y_interface", "z"), gi)
        st.v_quantity = quantity_wrap(st.v, ("x_interface", "y", "z"), gi)
        runs.append((st, comm, fv_setup, pt_adjust, set_omega, hyper, c2l, adjust, omega_updater, tr))
    snaps = [dict() for _ in range(6)]
    errors = []

    def work(t, st, comm, fv_setup, pt_adjust, set_omega, hyper, c2l, adjust, omega_updater, tr):
        try:
            fvd.compute_preamble(st, False, config, fv_setup, pt_adjust)
            snaps[t]["pre"] = {k: np.array(getattr(st, k)) for k in FV_STEP_FIELDS}
            fvd.post_remap(st, False, config, hyper, set_omega, omega_updater, tr.damping_coefficients.da_min)
            snaps[t]["post"] = {k: np.array(getattr(st, k)) for k in FV_STEP_FIELDS}
            fvd.wrapup(st, comm, adjust, c2l, False)
            snaps[t]["wrap"] = {k: np.array(getattr(st, k)) for k in FV_STEP_FIELDS}
        except BaseException as exc:  # surfaced after join
            errors.append(exc)
            raise

    threads = [threading.Thread(target=work, args=(t,) + r[:9] + (r[9],)) for t, r in enumerate(runs)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    # the fields each phase writes
    written = {"pre": ("q_con", "cvm", "pkz", "pt", "cappa", "dp1"), "post": ("omga",),
               "wrap": cases.WATER_NAMES + ("pt", "u", "v", "ua", "va")}
    out = {}
    for phase, names in written.items():
        for k in names:
            out[f"{phase}_{k}"] = np.stack([snaps[t][phase][k] for t in range(6)])
    return out, {"region": "full storage"}


REMAP_FIELDS = cases.REMAP_TRACERS + ("pt", "delp", "delz", "peln", "u", "v", "w", "ua", "va", "cappa", "q_con",
                                      "pkz", "pk", "pe", "ps", "qcld")


def run_remap(case, n, nz):
    """LagrangianToEulerian (remapping.py:205-628) tile by tile, built and
    called as DynamicalCore builds and calls it (fv_dynamics.py:380-386,
    483-519), on the last k_split step (last_step, no adiabatic init,
    consv_te 0); the fields it writes, over the compute domain and the
    extra row of the D-grid winds."""
    import fv3core._config as spec
    from fv3core.stencils.remapping import LagrangianToEulerian

    config = spec.RemappingConfig(sat_adjust=spec.SatAdjustConfig(**cases.SAT_ADJUST_CONFIG),
                                  **cases.remap_config(case))
    grid = cases.grid_for(n)
    S = rr.storage
    out = {k: [] for k in REMAP_FIELDS}
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        tr.activate()
        l2e = LagrangianToEulerian(tr.stencil_factory, config, tr.grid_data.area_64, len(cases.REMAP_TRACERS),
                                   case["pfull"])
        tracers = {k: S(case[k][t]) for k in cases.REMAP_TRACERS}
        st = {k: S(case[k][t]) for k in ("pt", "delp", "delz", "peln", "u", "v", "w", "ua", "va", "cappa",
                                         "q_con", "qcld", "pkz", "pk", "pe", "omga", "dp1")}
        for k in ("phis", "te0_2d", "ps", "wsd"):
            st[k] = S(case[k][t], origin=(3, 3))
        l2e(tracers, st["pt"], st["delp"], st["delz"], st["peln"], st["u"], st["v"], st["w"], st["ua"], st["va"],
            st["cappa"], st["q_con"], st["qcld"], st["pkz"], st["pk"], st["pe"], st["phis"], st["te0_2d"],
            st["ps"], st["wsd"], st["omga"], case["ak"], case["bk"], case["pfull"], st["dp1"], case["ptop"],
            cases.C.KAPPA, cases.C.ZVIR, True, 0.0, case["mdt"], case["mdt"], False, len(cases.REMAP_TRACERS))
        box = (slice(3, 3 + n + 1), slice(3, 3 + n + 1))
        for k in REMAP_FIELDS:
            out[k].append(np.array(tracers[k] if k in tracers else st[k])[box])
    return {k: np.stack(v) for k, v in out.items()}, {"region": "storage [3, 3 + n + 1) in i and j"}



STEP_OUT = {"u": (0, 1, 0), "v": (1, 0, 0), "w": (0, 0, 0), "delz": (0, 0, 0), "delp": (0, 0, 0), "pt": (0, 0, 0),
            "pe": (0, 0, 1), "pk": (0, 0, 1), "peln": (0, 0, 1), "pkz": (0, 0, 0), "q_con": (0, 0, 0),
            "cappa": (0, 0, 0), "omga": (0, 0, 0), "ua": (0, 0, 0), "va": (0, 0, 0)}


def run_step(case, n, nz):
    """DynamicalCore.step_dynamics (fv_dynamics.py:395-557) for one k_split
    step, composed as DynamicalCore._compute composes it from the
    reference's own classes and functions (built as DynamicalCore.__init__
    builds them, fv_dynamics.py:252-394): compute_preamble, then _dyn (the
    dp1 copy, AcousticDynamics, TracerAdvection of the eight tracers),
    LagrangianToEulerian, post_remap and wrapup; six tiles in lock step on
    threads.  DynamicalCore's own temporaries (te_2d, te0_2d, wsd, cappa,
    dp1, cvm, gz) start at zero.  Stored: the prognostic state on the
    compute domain (+1 on the staggered axes and interfaces) and ps."""
    import threading
    import types

    import fv3core._config as spec
    from fv3core.stencils import fv_dynamics as fvd
    from fv3core.stencils import moist_cv
    from fv3core.stencils.c2l_ord import CubedToLatLon
    from fv3core.stencils.del2cubed import HyperdiffusionDamping
    from fv3core.stencils.dyn_core import AcousticDynamics
    from fv3core.stencils.fvtp2d import FiniteVolumeTransport
    from fv3core.stencils.neg_adj3 import AdjustNegativeTracerMixingRatio
    from fv3core.stencils.remapping import LagrangianToEulerian
    from fv3core.stencils.tracer_2d_1l import TracerAdvection
    from fv3core.utils.grid import quantity_wrap

    grid = cases.grid_for(n)
    exchange = rr._Exchange()
    S = rr.storage
    acfg = spec.AcousticDynamicsConfig(
        **{**cases.ACOUSTIC_CONFIG, "n_split": int(case["n_split"])},
        riemann=spec.RiemannConfig(**cases.RIEMANN_CONFIG),
        d_grid_shallow_water=spec.DGridShallowWaterLagrangianDynamicsConfig(**cases.DSW_CONFIG),
    )
    rcfg = spec.RemappingConfig(sat_adjust=spec.SatAdjustConfig(**cases.SAT_ADJUST_CONFIG),
                                **dict(cases.REMAP_CONFIG, do_sat_adj=bool(case["do_sat_adj"])))
    config = types.SimpleNamespace(hydrostatic=False, rf_fast=True, tau=10.0, adiabatic=False, kord_tm=-9,
                                   nf_omega=1, nwat=6, moist_phys=True)
    nq = len(cases.REMAP_TRACERS)
    dims3 = ("x", "y", "z")
    runs = []
    for t in range(6):
        tr = rr.TileReference(grid, t, nz)
        tr.activate()
        tr.add_tracer_grid()
        comm = rr.ThreadComm(t, n, 3, exchange)
        sf, gi = tr.stencil_factory, tr.grid_indexing
        ak, bk, pfull = (S(case[k], origin=(0,)) for k in ("ak", "bk", "pfull"))
        phis = S(case["phis"][t], origin=(0, 0))
        o = types.SimpleNamespace()
        o.fv_setup = sf.from_origin_domain(moist_cv.fv_setup, externals={"nwat": 6, "moist_phys": True},
                                           origin=gi.origin_compute(), domain=gi.domain_compute())
        o.pt_adjust = sf.from_origin_domain(fvd.pt_adjust, origin=gi.origin_compute(), domain=gi.domain_compute())
        o.set_omega = sf.from_origin_domain(fvd.set_omega, origin=gi.origin_compute(), domain=gi.domain_compute())
        o.ad = AcousticDynamics(comm, sf, tr.grid_data, tr.damping_coefficients, 0, False, False, acfg, ak, bk,
                                pfull, phis)
        transport = FiniteVolumeTransport(sf, tr.grid_data, tr.damping_coefficients, 0, hord=8)
        o.adv = TracerAdvection(sf, transport, comm, nq)
        o.l2e = LagrangianToEulerian(sf, rcfg, tr.grid_data.area_64, nq, np.asarray(pfull))
        o.hyper = HyperdiffusionDamping(sf, tr.damping_coefficients, tr.grid_data.rarea, config.nf_omega)
        o.c2l = CubedToLatLon(sf, tr.grid_data, order=4)
        o.adjust = AdjustNegativeTracerMixingRatio(sf, False, False)
        spec_o = gi.get_quantity_halo_spec(gi.domain_full(add=(1, 1, 1)), gi.origin_compute(), dims=list(dims3),
                                           n_halo=3)
        o.omega_updater = comm.get_scalar_halo_updater([spec_o])
        st = types.SimpleNamespace()
        for name in tuple(cases.ACOUSTIC_STATE) + cases.STEP_TRACERS + ("ps",):
            arr = case[name][t]
            setattr(st, name, S(arr, origin=(3, 3) if arr.ndim == 2 else (3, 3, 0)))
        # DynamicalCore's temporaries (fvdyn_temporaries, fv_dynamics.py:172-190)
        m = case["delp"].shape[1]
        for name in ("te_2d", "te0_2d", "wsd"):
            setattr(st, name, S(np.zeros((m, m)), origin=(3, 3)))
        for name in ("cappa", "dp1", "cvm"):
            setattr(st, name, S(np.zeros((m, m, nz + 1))))
        for name, dims in ACOUSTIC_DIMS.items():
            setattr(st, name + "_quantity", quantity_wrap(getattr(st, name), dims, gi))
        st.omga_quantity = quantity_wrap(st.omga, dims3, gi)
        o.tracers = {k: quantity_wrap(getattr(st, k), dims3, gi) for k in cases.REMAP_TRACERS}
        st.ak, st.bk, st.pfull = ak, bk, pfull
        st.consv_te, st.do_adiabatic_init, st.bdt = 0.0, False, float(case["dt_atmos"])
        st.mdt, st.n_split, st.k_split, st.ptop, st.ks = float(case["dt_atmos"]), int(case["n_split"]), 1, \
            case["ptop"], case["ks"]
        st.akap = cases.C.KAPPA
        st.qcld_quantity = quantity_wrap(st.qcld, dims3, gi)
        runs.append((t, o, st, comm, tr))
    errors = []

    def work(t, o, st, comm, tr):
        try:
            fvd.compute_preamble(st, False, config, o.fv_setup, o.pt_adjust)
            st.n_map = 1
            # _dyn (fv_dynamics.py:535-557): dp1 = delp, the acoustic loop,
            # then the tracers with the accumulated fluxes
            st.dp1[:, :, :nz] = st.delp[:, :, :nz]
            o.ad(st)
            o.adv(o.tracers, st.dp1, st.mfxd, st.mfyd, st.cxd, st.cyd, st.mdt)
            o.l2e({k: q.storage for k, q in o.tracers.items()}, st.pt, st.delp, st.delz, st.peln, st.u, st.v,
                  st.w, st.ua, st.va, st.cappa, st.q_con, st.qcld, st.pkz, st.pk, st.pe, st.phis, st.te0_2d,
                  st.ps, st.wsd, st.omga, st.ak, st.bk, st.pfull, st.dp1, st.ptop, cases.C.KAPPA, cases.C.ZVIR,
                  True, st.consv_te, st.bdt / st.k_split, st.bdt, st.do_adiabatic_init, nq)
            fvd.post_remap(st, False, config, o.hyper, o.set_omega, o.omega_updater,
                           tr.damping_coefficients.da_min)
            fvd.wrapup(st, comm, o.adjust, o.c2l, False)
        except BaseException as exc:  # surfaced after join
            errors.append(exc)
            raise

    threads = [threading.Thread(target=work, args=r) for r in runs]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    h = 3
    out = {}
    for name, (di, dj, dk) in STEP_OUT.items():
        out[name] = np.stack([np.asarray(getattr(r[2], name)) for r in runs])[:, h:h + n + di, h:h + n + dj,
                                                                             :nz + dk]
    for name in cases.STEP_TRACERS:
        out[name] = np.stack([np.asarray(getattr(r[2], name)) for r in runs])[:, h:h + n, h:h + n, :nz]
    out["ps"] = np.stack([np.asarray(r[2].ps) for r in runs])[:, h:h + n, h:h + n]
    return out, {"region": "compute domain (+1 on staggered axes and interfaces)"}


def run_gnomonic_ed(case, n, nz):
    """The reference's grid_type 0 face (gnomonic_grid with
    global_gnomonic_ed, fv3core/grid/global_setup.py:15-85: corner lon/lat of
    the first tile's compute domain before rotation) and its own metric
    functions on it (gnomonic.py: great_circle_distance_along_axis for dx,
    dy; get_area; lon_lat_corner_to_cell_center).  fv3core.grid's package
    init needs fv3gfs-util's partitioner, which is absent, so the three
    modules load without it."""
    import types

    if "fv3core.grid" not in sys.modules:
        pkg = types.ModuleType("fv3core.grid")
        pkg.__path__ = [os.path.join(rr.reference_root(), "fv3core", "grid")]
        sys.modules["fv3core.grid"] = pkg
    from fv3core.grid import gnomonic as gn
    from fv3core.grid.global_setup import gnomonic_grid
    from fv3core.utils.global_constants import RADIUS

    lon = np.zeros((n + 1, n + 1))
    lat = np.zeros((n + 1, n + 1))
    gnomonic_grid(0, lon, lat, np)
    dx = gn.great_circle_distance_along_axis(lon, lat, RADIUS, np, axis=0)
    dy = gn.great_circle_distance_along_axis(lon, lat, RADIUS, np, axis=1)
    area = gn.get_area(lon, lat, RADIUS, np)
    lon_a, lat_a = gn.lon_lat_corner_to_cell_center(lon, lat, np)
    outputs = dict(lon=lon, lat=lat, dx=dx, dy=dy, area=area, lon_a=lon_a, lat_a=lat_a)
    # the angles of calculate_supergrid_cos_sin (geometry.py:163-215) at the
    # four edge midpoints of each cell, and the corner angle of
    # _calculate_more_trig_terms (geometry.py:326-352), with the
    # reference's spherical_cos and midpoints
    P = gn.lon_lat_to_xyz(lon, lat, np)
    A = gn.lon_lat_to_xyz(lon_a, lat_a, np)
    mid = gn.xyz_midpoint
    outputs["cos_sg1"] = gn.spherical_cos(mid(P[:-1, :-1], P[:-1, 1:]), A, P[:-1, 1:], np)
    outputs["cos_sg2"] = gn.spherical_cos(mid(P[:-1, :-1], P[1:, :-1]), P[1:, :-1], A, np)
    outputs["cos_sg3"] = gn.spherical_cos(mid(P[1:, :-1], P[1:, 1:]), A, P[1:, :-1], np)
    outputs["cos_sg4"] = gn.spherical_cos(mid(P[:-1, 1:], P[1:, 1:]), P[:-1, 1:], A, np)
    sg6 = gn.spherical_cos(P[:-1, :-1], P[1:, :-1], P[:-1, 1:], np)
    sg8 = gn.spherical_cos(P[1:, 1:], P[1:, :-1], P[:-1, 1:], np)
    outputs["cosa_interior"] = 0.5 * (sg8[:-1, :-1] + sg6[1:, 1:])
    return outputs, {"radius": RADIUS}


RUNNERS = {
    "acoustics": (run_acoustics, dict(n=12, nz=8, seed=41)),
    "d_sw": (run_d_sw, dict(n=12, nz=8, seed=31)),
    "c_sw": (run_c_sw, dict(n=12, nz=6, seed=21)),
    "riem_solver_c": (run_riem_solver_c, dict(n=12, nz=16, seed=11)),
    "acoustics_c12_l79": (run_acoustics_compute, dict(n=12, nz=79, seed=7, n_split=1)),
    "tracer_advection": (run_tracer_advection, dict(n=12, nz=8, seed=61)),
    "fv_step": (run_fv_step, dict(n=12, nz=8, seed=71)),
    "remap": (run_remap, dict(n=4, nz=79, seed=81)),
    "remap_kord10": (run_remap, dict(n=4, nz=30, seed=83)),
    "remap_kord8": (run_remap, dict(n=4, nz=30, seed=85)),
    "remap_satadj": (run_remap, dict(n=4, nz=79, seed=87)),
    "step": (run_step, dict(n=12, nz=12, seed=101)),
    "step_satadj": (run_step, dict(n=12, nz=12, seed=103)),
    # the plain FP64 C12 L79 substep on the reference's own grid (grid_type 0)
    "acoustics_c12_l79_ed": (run_acoustics_compute, dict(n=12, nz=79, seed=7, n_split=1, lattice="equidistant")),
    "gnomonic_ed_c12": (run_gnomonic_ed, dict(n=12, nz=1, seed=0)),
    "gnomonic_ed_c48": (run_gnomonic_ed, dict(n=48, nz=1, seed=0)),
}


def main(names):
    rr.import_reference()
    for name in names or list(RUNNERS):
        fn, kw = RUNNERS[name]
        t0 = time.time()
        kw = dict(kw)
        cases.LATTICE = kw.pop("lattice", "equiangular")
        case = cases.CASES[name](**kw)
        outputs, meta = fn(case, kw["n"], kw["nz"])
        meta["lattice"] = cases.LATTICE
        cases.LATTICE = "equiangular"
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **outputs, **{f"meta_{k}": v for k, v in meta.items()}, **{f"arg_{k}": v for k, v in kw.items()})
        print(f"{name}: {time.time() - t0:.1f}s -> {path} ({os.path.getsize(path) / 1e3:.0f} kB)")


if __name__ == "__main__":
    main(sys.argv[1:])
