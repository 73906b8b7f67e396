"""``compute_pkz_tempadjust`` — reference ``fv3core/stencils/temperature_adjust.py:8-44``
(a stencil the reference builds over levels [0, nk_heat_dissipation))."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class ComputePkzTempadjust:
    def __init__(self, stencil_factory, nk_heat_dissipation):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        self._nk = int(nk_heat_dissipation)

    def __call__(self, delp, delz, cappa, heat_source, pt, pkz, delt_time_factor):
        gi = self._gi
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        _lib.call_ctx(
            "fv3b_pkz_tempadjust", self._ctx, f3(delp, "delp"), f3(delz, "delz"), f3(cappa, "cappa"),
            f3(heat_source, "heat_source"), f3(pt, "pt"), f3(pkz, "pkz"), float(delt_time_factor), self._nk,
            stream_ptr(),
        )
