"""Run CUDA stages through the package's drop-in classes (shared by tests)."""
import functools

import numpy as np

import cases


@functools.lru_cache(maxsize=4)
def device_grid(n, nz):
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory

    gd = GridData(cases.grid_for(n), nz)
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    return gd, sf


def run_c_sw(case, n, nz, nord=3):
    import torch

    from fv3core_b200.stencils.c_sw import CGridShallowWaterDynamics
    from fv3core_b200.storage import to_device, to_host

    gd, sf = device_grid(n, nz)
    csw = CGridShallowWaterDynamics(sf, gd, False, 0, nord)
    names = ["delp", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "ut", "vt", "divgd", "omga"]
    dev = {k: to_device(case[k]) for k in names}
    delpc, ptc = csw(*[dev[k] for k in names], case["dt2"])
    torch.cuda.synchronize()
    out = {k: to_host(dev[k]) for k in names}
    out["delpc"] = to_host(delpc)
    out["ptc"] = to_host(ptc)
    return out


DSW_ARGS = ["delpc", "delp", "ptc", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "divgd", "mfx", "mfy",
            "cx", "cy", "crx", "cry", "xfx", "yfx", "q_con", "zh", "heat_source", "diss_est"]


def run_d_sw(case, n, nz, overrides=None):
    """``overrides``: namelist values replacing the baroclinic ones."""
    import dataclasses

    import torch

    from fv3core_b200.config import baroclinic_dsw_config
    from fv3core_b200.stencils.d_sw import DGridShallowWaterLagrangianDynamics
    from fv3core_b200.storage import to_device, to_host

    gd, sf = device_grid(n, nz)
    config = dataclasses.replace(baroclinic_dsw_config(), **(overrides or {}))
    dsw = DGridShallowWaterLagrangianDynamics(sf, gd, gd, None, False, False, config)
    dev = {k: to_device(case[k]) for k in DSW_ARGS}
    dsw(*[dev[k] for k in DSW_ARGS], case["dt"])
    torch.cuda.synchronize()
    return {k: to_host(dev[k]) for k in DSW_ARGS}


def make_acoustics(case, n, nz, precision="f64"):
    """(grid data, AcousticDynamics, device state) for a case of
    ``cases.acoustics_case``."""
    import types

    from fv3core_b200.config import (AcousticDynamicsConfig, DGridShallowWaterLagrangianDynamicsConfig,
                                     RiemannConfig)
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.halo import DeviceCubedSphereCommunicator
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.dyn_core import AcousticDynamics
    from fv3core_b200.storage import to_device

    gd = GridData(cases.grid_for(n), nz, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    cfg = AcousticDynamicsConfig(
        **{**cases.ACOUSTIC_CONFIG, "n_split": int(case["n_split"])},
        riemann=RiemannConfig(**cases.RIEMANN_CONFIG),
        d_grid_shallow_water=DGridShallowWaterLagrangianDynamicsConfig(**cases.DSW_CONFIG),
    )
    phis = to_device(case["phis"], dtype=dtype)
    ad = AcousticDynamics(DeviceCubedSphereCommunicator(gd.grid_indexing), sf, gd, gd, 0, False, False, cfg,
                          case["ak"], case["bk"], case["pfull"], phis)
    st = types.SimpleNamespace(**{k: to_device(case[k], dtype=dtype) for k in cases.ACOUSTIC_STATE})
    st.phis = phis
    for k in ("mdt", "n_map", "akap", "ptop", "ks"):
        setattr(st, k, case[k])
    return gd, ad, st


def run_acoustics(case, n, nz, precision="f64"):
    """The package's AcousticDynamics on a case of ``cases.acoustics_case``;
    returns the state and the driver's temporaries (prefixed ``tmp_``)."""
    import torch

    from fv3core_b200.storage import to_host

    gd, ad, st = make_acoustics(case, n, nz, precision)
    ad(st)
    torch.cuda.synchronize()
    out = {k: to_host(getattr(st, k)) for k in cases.ACOUSTIC_STATE}
    for name in ("gz", "zh", "pkc", "pk3", "heat_source", "divgd"):
        out["tmp_" + name] = to_host(ad.temporary(name).clone())
    gd.close()
    return out



def run_tracer_advection(case, n, nz, precision="f64"):
    """The package's TracerAdvection (hord_tr = 8 transport) on a case of
    ``cases.tracer_case``; returns the tracers and the in-place updated
    dp1, mfxd, mfyd, cxd, cyd."""
    import torch

    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.fvtp2d import FiniteVolumeTransport
    from fv3core_b200.stencils.tracer_2d_1l import TracerAdvection
    from fv3core_b200.storage import to_device, to_host

    gd = GridData(cases.grid_for(n), nz, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    try:
        transport = FiniteVolumeTransport(sf, gd, gd, 0, hord=8)
        ntr = case["tracers"].shape[0]
        adv = TracerAdvection(sf, transport, None, ntr)
        tracers = {f"q{q}": to_device(case["tracers"][q], dtype=dtype) for q in range(ntr)}
        dev = {k: to_device(case[k], dtype=dtype) for k in ("dp1", "mfxd", "mfyd", "cxd", "cyd")}
        adv(tracers, dev["dp1"], dev["mfxd"], dev["mfyd"], dev["cxd"], dev["cyd"], case["mdt"])
        torch.cuda.synchronize()
        out = {k: to_host(v) for k, v in dev.items()}
        out["tracers"] = np.stack([to_host(tracers[f"q{q}"]) for q in range(ntr)])
        transport.close()
        return out
    finally:
        gd.close()


def run_fv_step(case, n, nz, precision="f64"):
    """The package's compute_preamble, post_remap and wrapup on a case of
    ``cases.fv_step_case``; returns the state after each phase (prefixes
    pre_, post_, wrap_), as the oracle run does."""
    import types

    import torch

    from fv3core_b200.grid_data import GridData
    from fv3core_b200.halo import DeviceCubedSphereCommunicator, spec_for
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils import fv_dynamics as fvd
    from fv3core_b200.stencils.del2cubed import HyperdiffusionDamping
    from fv3core_b200.storage import to_device, to_host

    gd = GridData(cases.grid_for(n), nz, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    try:
        config = types.SimpleNamespace(hydrostatic=False, rf_fast=True, tau=10.0, adiabatic=False, kord_tm=-9,
                                       nf_omega=1)
        comm = DeviceCubedSphereCommunicator(gd.grid_indexing)
        st = types.SimpleNamespace(**{k: to_device(v, dtype=dtype) for k, v in case.items()})
        st.consv_te, st.do_adiabatic_init = 0.0, False
        out = {}

        def snap(prefix, names):
            torch.cuda.synchronize()
            out.update({f"{prefix}_{k}": to_host(getattr(st, k)) for k in names})

        fvd.compute_preamble(st, False, config, fvd.FvSetup(sf), fvd.PtAdjust(sf))
        snap("pre", ("q_con", "cvm", "pkz", "pt", "cappa", "dp1"))
        omega_updater = comm.get_scalar_halo_updater([spec_for(gd.grid_indexing, ("x", "y", "z"))])
        fvd.post_remap(st, False, config, HyperdiffusionDamping(sf, gd, gd.rarea, config.nf_omega),
                       fvd.SetOmega(sf), omega_updater, gd.da_min)
        snap("post", ("omga",))
        fvd.wrapup(st, comm, fvd.AdjustNegativeTracerMixingRatio(sf, False, False), fvd.CubedToLatLon(sf, gd, 4),
                   False)
        snap("wrap", cases.WATER_NAMES + ("pt", "u", "v", "ua", "va"))
        return out
    finally:
        gd.close()


def run_remap(case, n, nz, precision="f64"):
    """The package's LagrangianToEulerian on a case of ``cases.remap_case``
    (last step, no adiabatic init, consv_te 0); returns the remapped fields
    over the full storage."""
    import torch

    from fv3core_b200 import constants as C
    from fv3core_b200.config import RemappingConfig, SatAdjustConfig
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.remapping import LagrangianToEulerian
    from fv3core_b200.storage import to_device, to_host

    gd = GridData(cases.grid_for(n), nz, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    try:
        config = RemappingConfig(sat_adjust=SatAdjustConfig(**cases.SAT_ADJUST_CONFIG), **cases.remap_config(case))
        l2e = LagrangianToEulerian(sf, config, None, len(cases.REMAP_TRACERS), case["pfull"])
        dev = {k: to_device(case[k], dtype=dtype) for k in cases.REMAP_TRACERS + cases.REMAP_STATE
               + ("qcld", "omga", "dp1", "phis")}
        tracers = {k: dev[k] for k in cases.REMAP_TRACERS}
        d = dev
        l2e(tracers, d["pt"], d["delp"], d["delz"], d["peln"], d["u"], d["v"], d["w"], d["ua"], d["va"],
            d["cappa"], d["q_con"], d["qcld"], d["pkz"], d["pk"], d["pe"], d["phis"], d["te0_2d"], d["ps"],
            d["wsd"], d["omga"], case["ak"], case["bk"], case["pfull"], d["dp1"], case["ptop"], C.KAPPA, C.ZVIR,
            True, 0.0, case["mdt"], case["mdt"], False, len(cases.REMAP_TRACERS))
        torch.cuda.synchronize()
        return {k: to_host(dev[k]) for k in cases.REMAP_TRACERS + cases.REMAP_STATE + ("qcld",)}
    finally:
        gd.close()


def run_step(case, n, nz, precision="f64", steps=1):
    """The package's DynamicalCore.step_dynamics on a case of
    ``cases.step_case`` (``steps`` steps of dt_atmos); returns the full
    storages of the state."""
    import torch

    from fv3core_b200.config import DynamicalCoreConfig
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.fv_dynamics import DynamicalCore
    from fv3core_b200.storage import to_device, to_host

    gd = GridData(cases.grid_for(n), nz, precision=precision)
    dtype = gd.grid_indexing.dtype
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    try:
        config = DynamicalCoreConfig(**cases.dycore_namelist(n, nz, int(case["n_split"]),
                                                             bool(case.get("do_sat_adj", False))))
        phis = to_device(case["phis"], dtype=dtype)
        core = DynamicalCore(None, gd, sf, gd, config, case["ak"], case["bk"], phis)
        names = tuple(cases.ACOUSTIC_STATE) + cases.STEP_TRACERS + ("ps",)
        state = {k: to_device(case[k], dtype=dtype) for k in names if k not in ("phis",)}
        state["phis"] = phis
        for _ in range(steps):
            core.step_dynamics(state, False, False, float(case["dt_atmos"]), case["ptop"], int(case["n_split"]),
                               case["ks"])
        torch.cuda.synchronize()
        out = {k: to_host(v) for k, v in state.items()}
        # cappa is not a step_dynamics argument: the step keeps it in
        # DynamicalCore's own temporary, as the reference does
        out["cappa"] = to_host(core._temporaries["cappa"])
        return out
    finally:
        gd.close()
