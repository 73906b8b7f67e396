"""``DGridShallowWaterLagrangianDynamics`` — reference
``fv3core/stencils/d_sw.py:606-1131``."""
import ctypes

from .. import _lib
from ..storage import check_field, stream_ptr

ARG_NAMES = ("delpc", "delp", "ptc", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "divgd", "mfx", "mfy",
             "cx", "cy", "crx", "cry", "xfx", "yfx", "q_con", "zh", "heat_source", "diss_est")


class DGridShallowWaterLagrangianDynamics:
    """Fortran name d_sw: full-timestep advance of the D-grid winds, delp,
    pt, w and q_con (with flux preparation, PPM transport, del-n and
    divergence damping and the heat source)."""

    def __init__(self, stencil_factory, grid_data, damping_coefficients, column_namelist, nested, stretched_grid,
                 config):
        if config.grid_type >= 3:
            raise AssertionError("ubke and vbke only implemented for grid_type < 3")
        if config.inline_q:
            raise AssertionError("inline_q not yet implemented")
        if config.d_ext > 0:
            raise AssertionError("untested d_ext > 0. need to call a2b_ord2, not yet implemented")
        if nested or stretched_grid:
            raise NotImplementedError("nested and stretched grids are not supported")
        self._gi = stencil_factory.grid_indexing
        self.grid_data = grid_data
        c = _lib.DswConfig()
        for name, _ in _lib.DswConfig._fields_:
            setattr(c, name, type(getattr(c, name))(getattr(config, name)))
        self._config = c
        _lib.call_ctx("fv3b_d_sw_setup", grid_data.ctx, ctypes.addressof(c))

    def __call__(self, delpc, delp, ptc, pt, u, v, w, uc, vc, ua, va, divgd, mfx, mfy, cx, cy, crx, cry,
                 xfx, yfx, q_con, zh, heat_source, diss_est, dt):
        fields = (delpc, delp, ptc, pt, u, v, w, uc, vc, ua, va, divgd, mfx, mfy, cx, cy, crx, cry,
                  xfx, yfx, q_con, zh, heat_source, diss_est)
        ptrs = [check_field(f, self._gi, "3d", n) for f, n in zip(fields, ARG_NAMES)]
        _lib.call_ctx("fv3b_d_sw", self.grid_data.ctx, *ptrs, float(dt), stream_ptr())
