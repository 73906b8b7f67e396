"""``UpdateHeightOnDGrid`` — reference ``fv3core/stencils/updatedzd.py:189-393``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context, host_column


class UpdateHeightOnDGrid:
    """Advects the interface heights with the D-grid fluxes (interpolated to
    interfaces by a cubic spline), with PPM transport of order hord_tm and
    del-n damping, and sets the surface vertical velocity.

    The damping columns are the D-grid ones: build the
    DGridShallowWaterLagrangianDynamics of the same grid first (as the
    reference's AcousticDynamics does)."""

    def __init__(self, stencil_factory, damping_coefficients, grid_data, grid_type, hord_tm, dp0, column_namelist,
                 k_bounds=None):
        if grid_type >= 3:
            raise NotImplementedError("grid_type >= 3 is not implemented")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        dp = host_column(dp0, self._gi.npz + 1, "dp0")
        _lib.call_ctx("fv3b_update_dz_d_setup", self._ctx, dp.ctypes.data, int(hord_tm))

    def __call__(self, surface_height, height, courant_number_x, courant_number_y, x_area_flux, y_area_flux, ws,
                 dt):
        gi = self._gi
        _lib.call_ctx(
            "fv3b_update_dz_d", self._ctx,
            check_field(surface_height, gi, "2d", "surface_height"), check_field(height, gi, "3d", "height"),
            check_field(courant_number_x, gi, "3d", "courant_number_x"),
            check_field(courant_number_y, gi, "3d", "courant_number_y"),
            check_field(x_area_flux, gi, "3d", "x_area_flux"), check_field(y_area_flux, gi, "3d", "y_area_flux"),
            check_field(ws, gi, "2d", "ws"), float(dt), stream_ptr(),
        )
