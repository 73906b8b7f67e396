"""``p_grad_c_stencil`` — reference ``fv3core/stencils/dyn_core.py:101-145``
(a stencil the reference builds with ``stencil_factory.from_origin_domain``)."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context


class PGradC:
    """C-grid pressure-gradient update of uc, vc (nonhydrostatic form)."""

    def __init__(self, stencil_factory, hydrostatic=False):
        if hydrostatic:
            raise NotImplementedError("only the nonhydrostatic form is implemented")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)

    def __call__(self, rdxc, rdyc, uc, vc, delpc, pkc, gz, dt2):
        gi = self._gi
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        _lib.call_ctx("fv3b_p_grad_c", self._ctx, f3(uc, "uc"), f3(vc, "vc"), f3(delpc, "delpc"), f3(pkc, "pkc"),
                      f3(gz, "gz"), float(dt2), stream_ptr())
