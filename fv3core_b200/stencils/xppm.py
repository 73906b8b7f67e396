"""``XPiecewiseParabolic`` — reference ``fv3core/stencils/xppm.py:283-347``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class PiecewiseParabolic:
    """PPM flux along one axis over the box [origin, origin + domain)."""

    AXIS = 0

    def __init__(self, stencil_factory, dxa, grid_type, iord, origin, domain):
        if grid_type >= 3:
            raise AssertionError("grid_type >= 3 is not implemented")
        if iord not in (5, 6, 7, 8):
            raise NotImplementedError(f"iord={iord}: PPM orders 5, 6, 7 and 8 are implemented")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        # the grid's own cell widths (dxa / dya) live in the device context
        self._dxa = dxa
        self._iord = int(iord)
        self._origin = tuple(int(x) for x in origin)
        self._domain = tuple(int(x) for x in domain)
        if len(self._origin) != 3 or len(self._domain) != 3:
            raise ValueError("origin and domain must have three entries (i, j, k)")

    def __call__(self, q_in, c, q_mean_advected_through_interface):
        gi = self._gi
        (i0, j0, k0), (ni, nj, nk) = self._origin, self._domain
        _lib.call_ctx(
            "fv3b_ppm_flux", self._ctx, self.AXIS, self._iord, check_field(q_in, gi, "3d", "q_in"),
            check_field(c, gi, "3d", "c"),
            check_field(q_mean_advected_through_interface, gi, "3d", "q_mean_advected_through_interface"),
            i0, j0, k0, ni, nj, nk, stream_ptr(),
        )


class XPiecewiseParabolic(PiecewiseParabolic):
    """Fortran xppm: the mean value of q advected through each x-interface
    for Courant number c, by a piecewise-parabolic reconstruction of order
    iord (monotonic PPM for 5-7, the ord-8 limiter for 8)."""

    AXIS = 0
