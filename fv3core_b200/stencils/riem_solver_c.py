"""``RiemannSolverC`` — reference ``fv3core/stencils/riem_solver_c.py:67-165``."""
from .. import _lib
from ..storage import check_field, stream_ptr


class RiemannSolverC:
    """Fortran subroutine Riem_Solver_C: semi-implicit vertical sound-wave
    solve over dt2 on the C grid, for the columns one cell beyond the compute
    domain of every tile."""

    def __init__(self, stencil_factory, p_fac):
        self._gi = stencil_factory.grid_indexing
        self._p_fac = float(p_fac)
        self._dims = self._gi.dims()

    def __call__(self, dt2, cappa, ptop, hs, ws, ptc, q_con, delpc, gz, pef, w3):
        gi = self._gi
        _lib.call(
            "fv3b_riem_solver_c",
            self._dims,
            float(dt2),
            float(ptop),
            self._p_fac,
            check_field(cappa, gi, "3d", "cappa"),
            check_field(hs, gi, "2d", "hs"),
            check_field(ws, gi, "2d", "ws"),
            check_field(ptc, gi, "3d", "ptc"),
            check_field(q_con, gi, "3d", "q_con"),
            check_field(delpc, gi, "3d", "delpc"),
            check_field(gz, gi, "3d", "gz"),
            check_field(pef, gi, "3d", "pef"),
            check_field(w3, gi, "3d", "w3"),
            stream_ptr(),
            precision=gi.precision,
        )
