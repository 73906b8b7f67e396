"""``TracerAdvection`` — reference ``fv3core/stencils/tracer_2d_1l.py:120-300``."""
import ctypes

import torch

from .. import _lib
from ..storage import check_field, stream_ptr


class TracerAdvection:
    """Fortran tracer_2D_1L: horizontal advection of the tracers with the
    mass fluxes and Courant numbers the acoustic loop accumulated, in three
    sub-steps of ``transport`` (a FiniteVolumeTransport, hord_tr), with the
    tracer halo updates on the device.  ``comm`` is accepted for the
    reference's signature; the halo exchange is the library's own."""

    def __init__(self, stencil_factory, transport, comm, tracer_count):
        self._gi = stencil_factory.grid_indexing
        self._transport = transport
        self._tracer_count = int(tracer_count)
        self.comm = comm

    def __call__(self, tracers, dp1, mfxd, mfyd, cxd, cyd, mdt):
        """tracers: a mapping of names to fields (torch tensors in device
        layout, or quantities whose ``storage`` is one), updated in place.
        cxd, cyd, mfxd, mfyd are scaled by 1/3 in place and dp1 holds an
        intermediate pressure thickness afterwards, as in the reference."""
        if len(tracers) != self._tracer_count:
            raise ValueError(
                f"incorrect number of tracers, {self._tracer_count} was "
                f"specified on init but {len(tracers)} were passed"
            )
        gi = self._gi
        fields = [q if isinstance(q, torch.Tensor) else q.storage for q in tracers.values()]
        ptrs = (ctypes.c_void_p * max(1, len(fields)))(
            *[check_field(f, gi, "3d", f"tracer {name}") for name, f in zip(tracers, fields)]
        )
        _lib.call_precision(
            "fv3b_tracer_advection", gi.precision, self._transport.handle, len(fields), ptrs,
            check_field(dp1, gi, "3d", "dp1"), check_field(mfxd, gi, "3d", "mfxd"),
            check_field(mfyd, gi, "3d", "mfyd"), check_field(cxd, gi, "3d", "cxd"),
            check_field(cyd, gi, "3d", "cyd"), float(mdt), stream_ptr(),
        )
