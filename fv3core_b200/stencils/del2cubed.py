"""``HyperdiffusionDamping`` — reference ``fv3core/stencils/del2cubed.py:77-181``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class HyperdiffusionDamping:
    """Fortran name del2_cubed: min(3, nmax) passes of del-2 filtering."""

    def __init__(self, stencil_factory, damping_coefficients, rarea, nmax):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        self._nmax = int(nmax)

    def __call__(self, qdel, cd):
        _lib.call_ctx("fv3b_del2cubed", self._ctx, check_field(qdel, self._gi, "3d", "qdel"), float(cd),
                      self._nmax, stream_ptr())
