"""``FiniteVolumeTransport`` — reference ``fv3core/stencils/fvtp2d.py:151-362``."""
import ctypes
import dataclasses
from typing import Any

from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import context, host_column


@dataclasses.dataclass
class CopiedCorners:
    """The reference's container of a field and its corner-copied versions
    (fvtp2d.py:96-111).  Here only ``base`` is used: the transport copies the
    x-direction corners into it and reads the y-direction copies on the fly."""

    base: Any
    x_differentiable: Any = None
    y_differentiable: Any = None


class FiniteVolumeTransport:
    """Fortran fv_tp_2d: the Lin-Rood 2-D transport fluxes of a scalar
    (Putman and Lin 2007, eq. 16-17) with PPM of order ``hord`` (5, 6, 7, or
    8 for the ord-8 limiter of tracer transport) and optional del-n damping
    (``nord`` and ``damp_c`` per-level columns, both or neither)."""

    def __init__(self, stencil_factory, grid_data, damping_coefficients, grid_type, hord, nord=None, damp_c=None):
        if grid_type >= 3:
            raise AssertionError("grid_type >= 3 is not implemented (xppm.py:299)")
        if hord not in (5, 6, 7, 8):
            raise NotImplementedError(f"hord={hord}: PPM orders 5, 6, 7 and 8 are implemented")
        self._gi = stencil_factory.grid_indexing
        self._ctx = context(stencil_factory)
        self._precision = self._gi.precision
        self.hord = hord
        nk = self._gi.npz
        self._damped = nord is not None and damp_c is not None
        self._keep = []
        if self._damped:
            nord_h = host_column(nord, nk, "nord")
            damp_h = host_column(damp_c, nk, "damp_c")
            n = min(nord_h.shape[0], damp_h.shape[0])
            self._keep = [nord_h, damp_h]
            args = (nord_h.ctypes.data, damp_h.ctypes.data, n)
        else:
            args = (None, None, 0)
        tr = ctypes.c_void_p()
        _lib.call_ctx("fv3b_transport_create", self._ctx, int(hord), *args, ctypes.byref(tr))
        self._transport = tr

    @property
    def handle(self):
        """The C ABI's ``fv3b_transport*`` of this transport."""
        return self._transport

    def __call__(self, q, crx, cry, x_area_flux, y_area_flux, q_x_flux, q_y_flux, x_mass_flux=None,
                 y_mass_flux=None, mass=None):
        """q: a field, or a CopiedCorners whose base is the field; its
        cube-corner halo blocks take their x-direction copies, as the
        reference's base storage does."""
        if self._damped and mass is None and (x_mass_flux is not None or y_mass_flux is not None):
            raise ValueError("when damping is enabled, mass must be given if mass flux is given")
        gi = self._gi
        base = q.base if hasattr(q, "base") else q

        def opt(t, name):
            return None if t is None else check_field(t, gi, "3d", name)

        _lib.call_precision(
            "fv3b_fvtp2d", self._precision, self._transport, check_field(base, gi, "3d", "q"),
            check_field(crx, gi, "3d", "crx"), check_field(cry, gi, "3d", "cry"),
            check_field(x_area_flux, gi, "3d", "x_area_flux"), check_field(y_area_flux, gi, "3d", "y_area_flux"),
            check_field(q_x_flux, gi, "3d", "q_x_flux"), check_field(q_y_flux, gi, "3d", "q_y_flux"),
            opt(x_mass_flux, "x_mass_flux"), opt(y_mass_flux, "y_mass_flux"), opt(mass, "mass"), stream_ptr(),
        )

    def close(self):
        if getattr(self, "_transport", None) is not None and self._transport.value:
            _lib.lib(self._precision).fv3b_transport_destroy(self._transport)
            self._transport = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
