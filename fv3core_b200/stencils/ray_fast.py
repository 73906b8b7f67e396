"""``RayleighDamping`` — reference ``fv3core/stencils/ray_fast.py:131-192``."""
from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context, host_column


class RayleighDamping:
    """Fast Rayleigh friction of u, v (and w) on the levels above
    rf_cutoff, with the removed momentum given back to the layers above
    rf_cutoff + min(100, 10 ptop).  dp and pfull are K fields; they are read
    on the host (the per-level factors are computed there)."""

    def __init__(self, stencil_factory, rf_cutoff, tau, hydrostatic):
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        self._rf_cutoff = float(rf_cutoff)
        self._tau = float(tau)
        self._hydrostatic = 1 if hydrostatic else 0

    def __call__(self, u, v, w, dp, pfull, dt, ptop, ks):
        gi = self._gi
        npz = gi.npz
        dp_h = host_column(dp, npz, "dp")
        pf_h = host_column(pfull, npz, "pfull")
        _lib.call_ctx(
            "fv3b_ray_fast", self._ctx, check_field(u, gi, "3d", "u"), check_field(v, gi, "3d", "v"),
            check_field(w, gi, "3d", "w"), dp_h.ctypes.data, pf_h.ctypes.data, float(dt), float(ptop),
            self._rf_cutoff, self._tau, self._hydrostatic, stream_ptr(),
        )
