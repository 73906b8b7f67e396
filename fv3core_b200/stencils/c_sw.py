"""``CGridShallowWaterDynamics`` — reference ``fv3core/stencils/c_sw.py:379-659``."""
import torch

from .. import _lib
from ..storage import check_field, empty, stream_ptr


class CGridShallowWaterDynamics:
    """Fortran name c_sw: advances the C-grid winds by half a time step and
    produces delpc, ptc, omga, divgd (the D->A->C interpolation of
    d2a2c_vect included)."""

    def __init__(self, stencil_factory, grid_data, nested, grid_type, nord):
        if grid_type >= 3:
            raise NotImplementedError("unimplemented grid_type >= 3")
        if nested:
            raise NotImplementedError("nested grids are not supported")
        self._gi = stencil_factory.grid_indexing
        self.grid_data = grid_data
        self._nord = int(nord)
        self.delpc = empty(self._gi, "3d").fill_(float("nan"))
        self.ptc = empty(self._gi, "3d").fill_(float("nan"))

    def __call__(self, delp, pt, u, v, w, uc, vc, ua, va, ut, vt, divgd, omga, dt2):
        gi = self._gi
        names = ("delp", "pt", "u", "v", "w", "uc", "vc", "ua", "va", "ut", "vt", "divgd", "omga")
        ptrs = [check_field(f, gi, "3d", n) for f, n in zip((delp, pt, u, v, w, uc, vc, ua, va, ut, vt, divgd, omga), names)]
        _lib.call_ctx(
            "fv3b_c_sw", self.grid_data.ctx, *ptrs, float(dt2), self._nord,
            self.delpc.data_ptr(), self.ptc.data_ptr(), stream_ptr(),
        )
        return self.delpc, self.ptc
