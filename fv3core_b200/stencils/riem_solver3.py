"""``RiemannSolver3`` — reference ``fv3core/stencils/riem_solver3.py:106-242``."""
from .. import _lib
from ..storage import check_field, stream_ptr


class RiemannSolver3:
    """Fortran subroutine Riem_Solver3: the semi-implicit vertical
    sound-wave solve after the D-grid step, on the compute domain."""

    def __init__(self, stencil_factory, config):
        if config.a_imp <= 0.999:
            raise NotImplementedError("a_imp <= 0.999 is not implemented")
        if config.use_logp:
            raise NotImplementedError("use_logp=True is not implemented")
        if config.beta != 0:
            raise NotImplementedError("beta != 0 is not implemented")
        self._gi = stencil_factory.grid_indexing
        self._dims = self._gi.dims()
        self._p_fac = float(config.p_fac)

    def __call__(self, last_call, dt, cappa, ptop, zs, wsd, delz, q_con, delp, pt, zh, pe, ppe, pk3, pk, peln, w):
        gi = self._gi
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        _lib.call(
            "fv3b_riem_solver3", self._dims, 1 if last_call else 0, float(dt), float(ptop), self._p_fac,
            f3(cappa, "cappa"), check_field(zs, gi, "2d", "zs"), check_field(wsd, gi, "2d", "wsd"),
            f3(delz, "delz"), f3(q_con, "q_con"), f3(delp, "delp"), f3(pt, "pt"), f3(zh, "zh"), f3(pe, "pe"),
            f3(ppe, "ppe"), f3(pk3, "pk3"), f3(pk, "pk"), f3(peln, "peln"), f3(w, "w"), stream_ptr(),
            precision=gi.precision,
        )
