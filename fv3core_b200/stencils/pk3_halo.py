"""``PK3Halo`` — reference ``fv3core/stencils/pk3_halo.py:24-68``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class PK3Halo:
    """pk3 = p^akap on the two-cell ring around the compute domain."""

    def __init__(self, stencil_factory):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)

    def __call__(self, pk3, delp, ptop, akap):
        gi = self._gi
        _lib.call_ctx("fv3b_pk3_halo", self._ctx, check_field(pk3, gi, "3d", "pk3"),
                      check_field(delp, gi, "3d", "delp"), float(ptop), float(akap), stream_ptr())
