"""LagrangianToEulerian — reference ``fv3core/stencils/remapping.py:205-628``:
the vertical remapping of the deformed Lagrangian layers back onto the
hybrid-coordinate (Eulerian) levels, with the reference's constructor and
call signature.  The work runs in ``fv3b_lagrangian_to_eulerian``."""
import ctypes

from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context, host_column

CONSV_MIN = 0.001  # remapping.py:30


class LagrangianToEulerian:
    """Fortran Lagrangian_to_Eulerian (remapping.py:205-628).

    ``config`` is a RemappingConfig; with do_sat_adj the fast saturation
    adjustment runs after the remaps on the levels from kmp (the first
    level whose reference pressure ``pfull`` exceeds 10 hPa) down, with the
    grid's cell areas (``area_64`` is taken for the signature; the context
    holds the areas).  Rejects what the reference rejects: kord_tm >= 0 and
    hydrostatic."""

    def __init__(self, stencil_factory, config, area_64, nq, pfull):
        if config.kord_tm >= 0:
            raise NotImplementedError("map ppm, untested mode where kord_tm >= 0")
        if config.hydrostatic:
            raise NotImplementedError("Hydrostatic is not implemented")
        for name in ("kord_tm", "kord_tr", "kord_wz", "kord_mt"):
            if abs(getattr(config, name)) > 10:
                raise AssertionError(f"kord {getattr(config, name)} not implemented.")
        if nq != len(_lib.REMAP_TRACERS):
            raise NotImplementedError(f"nq={nq}: the remapping is built for the {len(_lib.REMAP_TRACERS)} tracers "
                                      "DynamicalCore advects")
        gi = stencil_factory.grid_indexing
        self._gi = gi
        self._ctx = context(stencil_factory)
        self._nq = nq
        self._t_min = 184.0
        npz = gi.domain[2]
        self._pfull = host_column(pfull, npz, "pfull")
        self._config = _lib.RemapConfig(int(config.kord_tm), int(config.kord_tr), int(config.kord_wz),
                                        int(config.kord_mt), int(bool(config.fill)), 0)
        self._akbk = None
        self._sat = None
        if config.do_sat_adj:
            sa = config.sat_adjust
            self._sat = _lib.SatAdjustConfig(*([float(getattr(sa, n)) for n in _lib.SAT_ADJUST_DOUBLES]
                                               + [int(getattr(sa, n)) for n in _lib.SAT_ADJUST_INTS]))
        # kmp (remapping.py:396-400): the first level below 10 hPa
        self.kmp = npz - 1
        for k in range(self._pfull.shape[0]):
            if self._pfull[k] > 10.0e2:
                self.kmp = k
                break

    def _setup(self, ak, bk):
        npz = self._gi.domain[2]
        ak = host_column(ak, npz + 1, "ak")
        bk = host_column(bk, npz + 1, "bk")
        key = (ak.tobytes(), bk.tobytes())
        if key != self._akbk:
            _lib.call_ctx("fv3b_remap_setup", self._ctx, ak.ctypes.data, bk.ctypes.data)
            self._akbk = key

    def __call__(self, tracers, pt, delp, delz, peln, u, v, w, ua, va, cappa, q_con, q_cld, pkz, pk, pe, hs,
                 te0_2d, ps, wsd, omga, ak, bk, pfull, dp1, ptop, akap, zvir, last_step, consv_te, mdt, bdt,
                 do_adiabatic_init, nq):
        """remapping.py:416-628.  ``tracers`` maps the tracer names
        (qvapor, qliquid, qrain, qice, qsnow, qgraupel, qo3mr, qsgs_tke) to
        device fields; every other field is a device field in the library's
        layout (hs, te0_2d, ps, wsd 2-D).  q_cld, hs, dp1 and mdt feed the
        saturation adjustment (do_sat_adj); te0_2d, omga and bdt only the
        total-energy fixer and the omega remap, which the reference does not
        run either (consv_te 0, do_omega off)."""
        if last_step and not do_adiabatic_init:
            if consv_te > CONSV_MIN:
                raise NotImplementedError("We do not support consv_te > 0.001 because that would trigger an "
                                          "allReduce")
            if consv_te < -CONSV_MIN:
                raise NotImplementedError(f"Unimplemented/untested case consv({consv_te})  < -CONSV_MIN("
                                          f"{-CONSV_MIN})")
        gi = self._gi
        self._setup(ak, bk)
        f = _lib.RemapFields()
        for n, name in enumerate(_lib.REMAP_TRACERS):
            if name not in tracers:
                raise KeyError(f"tracers: missing {name}")
            f.tracers[n] = check_field(tracers[name], gi, "3d", name)
        fields = dict(pt=pt, delp=delp, delz=delz, peln=peln, u=u, v=v, w=w, ua=ua, va=va, cappa=cappa,
                      q_con=q_con, pkz=pkz, pk=pk, pe=pe)
        for name, t in fields.items():
            setattr(f, name, check_field(t, gi, "3d", name))
        f.ps = check_field(ps, gi, "2d", "ps")
        f.wsd = check_field(wsd, gi, "2d", "wsd")
        sat = None
        if self._sat is not None:
            f.qcld = check_field(q_cld, gi, "3d", "q_cld")
            f.dp1 = check_field(dp1, gi, "3d", "dp1")
            f.hs = check_field(hs, gi, "2d", "hs")
            sat = ctypes.addressof(self._sat)
        _lib.call_ctx("fv3b_lagrangian_to_eulerian", self._ctx, ctypes.addressof(f), ctypes.addressof(self._config),
                      sat, float(ptop), float(akap), float(zvir), float(mdt), int(self.kmp), int(bool(last_step)),
                      stream_ptr())
