"""The step preamble and epilogue of ``DynamicalCore.step_dynamics`` —
reference ``fv3core/stencils/fv_dynamics.py:32-169``: ``compute_preamble``,
``post_remap`` and ``wrapup`` with the reference's signatures, and the stencil
objects they take."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class FvSetup:
    """moist_cv.fv_setup (moist_cv.py:197-228) on the compute domain, built
    as DynamicalCore.__init__ builds it (fv_dynamics.py:320-328)."""

    def __init__(self, stencil_factory, nwat=6, moist_phys=True):
        if not moist_phys:
            raise AssertionError("fvsetup is only implemented for moist_phys=true")
        if nwat != 6:
            raise AssertionError("Only nwat=6 has been implemented and tested")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)


class PtAdjust:
    """pt_adjust (fv_dynamics.py:32-34) on the compute domain; runs inside
    compute_preamble's pass together with fv_setup."""

    def __init__(self, stencil_factory):
        self._gi = stencil_factory.grid_indexing


class SetOmega:
    """set_omega (fv_dynamics.py:37-39) on the compute domain."""

    def __init__(self, stencil_factory):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)


def compute_preamble(state, is_root_rank, config, fv_setup_stencil, pt_adjust_stencil):
    """fv_dynamics.py:54-106.  ``state`` carries qvapor ... qgraupel, q_con,
    cvm, pkz, pt, cappa, delp, delz, dp1 (device fields) and the scalars
    consv_te and do_adiabatic_init."""
    if config.hydrostatic:
        raise NotImplementedError("Hydrostatic is not implemented")
    if state.consv_te > 0 and not state.do_adiabatic_init:
        raise NotImplementedError("compute total energy is not implemented, it needs an allReduce")
    if (not config.rf_fast) and config.tau != 0:
        raise NotImplementedError("Rayleigh_Super, called when rf_fast=False and tau !=0")
    if config.adiabatic and config.kord_tm > 0:
        raise NotImplementedError("unimplemented namelist options adiabatic with positive kord_tm")
    gi = fv_setup_stencil._gi
    names = ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "q_con", "cvm", "pkz", "pt", "cappa",
             "delp", "delz", "dp1")
    _lib.call_ctx("fv3b_compute_preamble", fv_setup_stencil._ctx,
                  *[check_field(getattr(state, n), gi, "3d", n) for n in names], stream_ptr())


def post_remap(state, is_root_rank, config, hyperdiffusion, set_omega_stencil, omega_halo_updater, da_min):
    """fv_dynamics.py:109-133: omga from w, then (nf_omega > 0) its halo
    update and del-2 filter with 0.18 da_min."""
    if not config.hydrostatic:
        gi = set_omega_stencil._gi
        _lib.call_ctx("fv3b_post_remap", set_omega_stencil._ctx,
                      *[check_field(getattr(state, n), gi, "3d", n) for n in ("delp", "delz", "w", "omga")], 0,
                      stream_ptr())
    if config.nf_omega > 0:
        omega_halo_updater.update([state.omga])
        hyperdiffusion(state.omga, 0.18 * da_min)


def wrapup(state, comm, adjust_stencil, cubed_to_latlon_stencil, is_root_rank):
    """fv_dynamics.py:136-169: the negative-tracer fixes, then the A-grid
    longitude / latitude winds."""
    adjust_stencil(state.qvapor, state.qliquid, state.qrain, state.qsnow, state.qice, state.qgraupel, state.qcld,
                   state.pt, state.delp, state.delz, state.peln)
    cubed_to_latlon_stencil(state.u, state.v, state.ua, state.va, comm)


class AdjustNegativeTracerMixingRatio:
    """Fortran neg_adj3 (neg_adj3.py:293-372): removes negative water
    species by borrowing from the other species and from the neighbouring
    levels."""

    def __init__(self, stencil_factory, check_negative, hydrostatic):
        if check_negative:
            raise NotImplementedError("Unimplemented namelist value check_negative=True")
        if hydrostatic:
            raise NotImplementedError("Unimplemented namelist hydrostatic=True")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)

    def __call__(self, qvapor, qliquid, qrain, qsnow, qice, qgraupel, qcld, pt, delp, delz, peln):
        gi = self._gi
        fields = dict(qvapor=qvapor, qliquid=qliquid, qrain=qrain, qsnow=qsnow, qice=qice, qgraupel=qgraupel,
                      qcld=qcld, pt=pt, delp=delp, delz=delz, peln=peln)
        _lib.call_ctx("fv3b_adjust_negative_tracers", self._ctx,
                      *[check_field(f, gi, "3d", n) for n, f in fields.items()], 0, stream_ptr())


class CubedToLatLon:
    """Fortran c2l_ord2 / c2l_ord4 (c2l_ord.py:75-141): D-grid winds to
    A-grid winds in longitude / latitude components.  ``grid_data`` must
    carry the transformation coefficients a11, a12, a21, a22 (device 2-D
    fields), as the reference's legacy grid does."""

    def __init__(self, stencil_factory, grid_data, order):
        if order not in (2, 4):
            raise ValueError("order must be 2 or 4")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        self._order = int(order)
        self._a = [getattr(grid_data, n) for n in ("a11", "a12", "a21", "a22")]

    def __call__(self, u, v, ua, va, comm=None):
        """``comm`` is accepted for the reference's signature: the order-4
        halo update of u and v runs on the device as part of this call."""
        gi = self._gi
        _lib.call_ctx("fv3b_cubed_to_latlon", self._ctx, check_field(u, gi, "3d", "u"), check_field(v, gi, "3d", "v"),
                      *[check_field(a, gi, "2d", n) for a, n in zip(self._a, ("a11", "a12", "a21", "a22"))],
                      check_field(ua, gi, "3d", "ua"), check_field(va, gi, "3d", "va"), self._order, stream_ptr())


# ---------------------------------------------------------------- the step
NQ = 8  # fv_dynamics.py:29, the tracers advected and remapped
TRACERS = _lib.REMAP_TRACERS  # utils.tracer_variables[0:NQ]


def init_pfull(ak, bk, p_ref):
    """init_pfull (fv_dynamics.py:42-51): layer-mean reference pressure of
    a column at surface pressure p_ref, (ph2 - ph1) / log(ph2 / ph1)."""
    import numpy as np

    ak = np.asarray(ak, dtype=np.float64)
    bk = np.asarray(bk, dtype=np.float64)
    ph1 = ak[:-1] + bk[:-1] * p_ref
    ph2 = ak[1:] + bk[1:] * p_ref
    return (ph2 - ph1) / np.log(ph2 / ph1)


def _get(state, name):
    if isinstance(state, dict):
        return state[name]
    return getattr(state, name)


class DynamicalCore:
    """fv_dynamics (fv_dynamics.py:193-557): one dynamics step of the
    nonhydrostatic core — preamble, k_split x (acoustic substeps, tracer
    advection, vertical remapping), the omega filter, the negative-tracer
    fixes and the A-grid winds — built as the reference builds it from its
    stage classes, each running as this library's kernels.

    ``comm``: a DeviceCubedSphereCommunicator (one is made when None);
    ``grid_data`` / ``damping_coefficients``: the GridData of
    ``stencil_factory``'s grid; ``ak``, ``bk``: host or device columns of
    npz+1 values; ``phis``: 2-D device field.  Not built (rejected at
    construction): the saturation adjustment (do_sat_adj) and what the
    reference rejects."""

    def __init__(self, comm, grid_data, stencil_factory, damping_coefficients, config, ak, bk, phis):
        import torch

        from .. import storage
        from ..halo import DeviceCubedSphereCommunicator, spec_for
        from ._common import host_column
        from .del2cubed import HyperdiffusionDamping
        from .dyn_core import AcousticDynamics
        from .fvtp2d import FiniteVolumeTransport
        from .remapping import LagrangianToEulerian
        from .tracer_2d_1l import TracerAdvection

        if not config.moist_phys:
            raise AssertionError("fvsetup is only implemented for moist_phys=true")
        if config.nwat != 6:
            raise AssertionError("Only nwat=6 has been implemented and tested")
        if config.inline_q or NQ == 0:
            raise NotImplementedError("tracer_2d not implemented, turn on z_tracer")
        gi = stencil_factory.grid_indexing
        self.grid_indexing = gi
        self.grid_data = grid_data
        self.config = config
        self.comm = comm if comm is not None else DeviceCubedSphereCommunicator(gi)
        self._da_min = damping_coefficients.da_min
        npz = gi.domain[2]
        self._ak = host_column(ak, npz + 1, "ak")
        self._bk = host_column(bk, npz + 1, "bk")
        self._phis = phis
        self._pfull = init_pfull(self._ak[:npz + 1], self._bk[:npz + 1], config.p_ref)
        self._fv_setup_stencil = FvSetup(stencil_factory, config.nwat, config.moist_phys)
        self._pt_adjust_stencil = PtAdjust(stencil_factory)
        self._set_omega_stencil = SetOmega(stencil_factory)
        transport = FiniteVolumeTransport(stencil_factory, grid_data, damping_coefficients, config.grid_type,
                                          hord=config.hord_tr)
        self.tracer_advection = TracerAdvection(stencil_factory, transport, self.comm, NQ)
        self.acoustic_dynamics = AcousticDynamics(self.comm, stencil_factory, grid_data, damping_coefficients,
                                                  config.grid_type, False, False, config.acoustic_dynamics,
                                                  self._ak, self._bk, self._pfull, phis)
        self._hyperdiffusion = HyperdiffusionDamping(stencil_factory, damping_coefficients, grid_data.rarea,
                                                     config.nf_omega)
        self._cubed_to_latlon = CubedToLatLon(stencil_factory, grid_data, order=config.c2l_ord)
        self._adjust_tracer_mixing_ratio = AdjustNegativeTracerMixingRatio(stencil_factory, config.check_negative,
                                                                           config.hydrostatic)
        self._lagrangian_to_eulerian_obj = LagrangianToEulerian(
            stencil_factory, config.remapping, getattr(grid_data, "area_64", None), NQ, self._pfull)
        self._omega_halo_updater = self.comm.get_scalar_halo_updater([spec_for(gi, ("x", "y", "z"))])
        # fvdyn_temporaries (fv_dynamics.py:172-190): kept between steps
        self._temporaries = {name: storage.zeros(gi, "2d") for name in ("te_2d", "te0_2d", "wsd")}
        for name in ("cappa", "dp1", "cvm"):
            self._temporaries[name] = storage.zeros(gi, "3d")
        self._temporaries["gz"] = torch.zeros(gi.max_shape[2], dtype=gi.dtype, device="cuda")

    def step_dynamics(self, state, conserve_total_energy, do_adiabatic_init, timestep, ptop, n_split, ks,
                      timer=None):
        """fv_dynamics.py:395-428.  ``state`` maps (or has as attributes)
        the arg_specs names (fv_dynamics.py:198-250) to device fields:
        qvapor, qliquid, qrain, qsnow, qice, qgraupel, qo3mr, qsgs_tke,
        qcld, pt, delp, delz, peln, u, v, w, ua, va, uc, vc, q_con, pe, phis,
        pk, pkz, ps, omga, mfxd, mfyd, cxd, cyd, diss_estd (ak and bk are
        the constructor's).  Every field is updated in place."""
        import types

        names = TRACERS + ("qcld", "pt", "delp", "delz", "peln", "u", "v", "w", "ua", "va", "uc", "vc", "q_con",
                           "pe", "phis", "pk", "pkz", "ps", "omga", "mfxd", "mfyd", "cxd", "cyd", "diss_estd")
        st = types.SimpleNamespace(**{name: _get(state, name) for name in names})
        st.__dict__.update(
            consv_te=conserve_total_energy, bdt=timestep, mdt=timestep / self.config.k_split,
            do_adiabatic_init=do_adiabatic_init, ptop=ptop, n_split=n_split, k_split=self.config.k_split, ks=ks,
        )
        self._compute(st)

    def _compute(self, state):
        """fv_dynamics.py:430-533."""
        from ..constants import KAPPA, ZVIR

        state.__dict__.update(self._temporaries)
        tracers = {name: getattr(state, name) for name in TRACERS}
        state.ak, state.bk = self._ak, self._bk
        state.akap = KAPPA
        compute_preamble(state, True, self.config, self._fv_setup_stencil, self._pt_adjust_stencil)
        npz = self.grid_indexing.domain[2]
        for n_map in range(state.k_split):
            state.n_map = n_map + 1
            last_step = n_map == state.k_split - 1
            self._dyn(state, tracers)
            if npz > 4:
                self._lagrangian_to_eulerian_obj(
                    tracers, state.pt, state.delp, state.delz, state.peln, state.u, state.v, state.w, state.ua,
                    state.va, state.cappa, state.q_con, state.qcld, state.pkz, state.pk, state.pe, state.phis,
                    state.te0_2d, state.ps, state.wsd, state.omga, self._ak, self._bk, self._pfull, state.dp1,
                    state.ptop, KAPPA, ZVIR, last_step, state.consv_te, state.bdt / state.k_split, state.bdt,
                    state.do_adiabatic_init, NQ)
                if last_step:
                    post_remap(state, True, self.config, self._hyperdiffusion, self._set_omega_stencil,
                               self._omega_halo_updater, self._da_min)
        wrapup(state, self.comm, self._adjust_tracer_mixing_ratio, self._cubed_to_latlon, True)

    def _dyn(self, state, tracers):
        """fv_dynamics.py:535-557: dp1 = delp on the npz layers, the acoustic
        substeps, then the tracers with the accumulated fluxes."""
        npz = self.grid_indexing.domain[2]
        state.dp1[:, :npz].copy_(state.delp[:, :npz])
        self.acoustic_dynamics(state)
        if self.config.z_tracer:
            self.tracer_advection(tracers, state.dp1, state.mfxd, state.mfyd, state.cxd, state.cyd, state.mdt)
