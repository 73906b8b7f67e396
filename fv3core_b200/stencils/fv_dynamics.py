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
