"""``UpdateGeopotentialHeightOnCGrid`` — reference
``fv3core/stencils/updatedzc.py:123-163``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class UpdateGeopotentialHeightOnCGrid:
    """Advects the interface heights gz with the C-grid fluxes over dt and
    sets the surface vertical velocity ws (one cell beyond the compute
    domain)."""

    def __init__(self, stencil_factory, area):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)

    def __call__(self, dp_ref, zs, ut, vt, gz, ws, dt):
        gi = self._gi
        _lib.call_ctx(
            "fv3b_update_dz_c", self._ctx,
            check_field(dp_ref, gi, "1d", "dp_ref"), check_field(zs, gi, "2d", "zs"),
            check_field(ut, gi, "3d", "ut"), check_field(vt, gi, "3d", "vt"),
            check_field(gz, gi, "3d", "gz"), check_field(ws, gi, "2d", "ws"), float(dt), stream_ptr(),
        )
