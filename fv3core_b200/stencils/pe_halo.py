"""``edge_pe`` — reference ``fv3core/stencils/pe_halo.py:6-33`` (a stencil
the reference builds with ``stencil_factory.from_origin_domain``)."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class EdgePe:
    """Interface pressure on the one-cell ring around the compute domain."""

    def __init__(self, stencil_factory):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)

    def __call__(self, pe, delp, ptop):
        gi = self._gi
        _lib.call_ctx("fv3b_edge_pe", self._ctx, check_field(pe, gi, "3d", "pe"), check_field(delp, gi, "3d", "delp"),
                      float(ptop), stream_ptr())
