"""``YPiecewiseParabolic`` — reference ``fv3core/stencils/yppm.py`` (xppm.py
with the axes exchanged)."""
from .xppm import PiecewiseParabolic


class YPiecewiseParabolic(PiecewiseParabolic):
    """Fortran yppm: the mean value of q advected through each y-interface
    for Courant number c (constructor argument ``dya``, order ``jord``)."""

    AXIS = 1

    def __init__(self, stencil_factory, dya, grid_type, jord, origin, domain):
        super().__init__(stencil_factory, dya, grid_type, jord, origin, domain)
