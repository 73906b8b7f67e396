"""``NonHydrostaticPressureGradient`` — reference ``fv3core/stencils/nh_p_grad.py:71-206``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class NonHydrostaticPressureGradient:
    """Updates the D-grid winds with the hydrostatic and nonhydrostatic
    pressure-gradient forces (pp, pk3, gz replaced by their B-grid values)."""

    def __init__(self, stencil_factory, grid_data, grid_type):
        if grid_type >= 3:
            raise NotImplementedError("grid_type >= 3 is not implemented")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)

    def __call__(self, u, v, pp, gz, pk3, delp, dt, ptop, akap):
        gi = self._gi
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        _lib.call_ctx(
            "fv3b_nh_p_grad", self._ctx, f3(u, "u"), f3(v, "v"), f3(pp, "pp"), f3(gz, "gz"), f3(pk3, "pk3"),
            f3(delp, "delp"), float(dt), float(ptop), float(akap), stream_ptr(),
        )
