"""On-device cubed-sphere halo updates with fv3gfs-util's interface.

The reference's AcousticDynamics receives a ``CubedSphereCommunicator``
(fv3gfs-util, one MPI rank per tile) and builds halo updaters from quantity
halo specs (fv3core/stencils/dyn_core.py:216-286).  Here all six tiles live in
one device array, so ``DeviceCubedSphereCommunicator`` needs no messages:
``start`` enqueues the gather kernel on the current stream and ``wait`` does
nothing (stream order already guarantees the data is ready for the next
kernel).
"""
from . import _lib
from .storage import stream_ptr

X_INTERFACE_DIM = "x_interface"
Y_INTERFACE_DIM = "y_interface"
Z_INTERFACE_DIM = "z_interface"


class HaloSpec:
    """What a halo update needs to know of a quantity: its staggering,
    halo width and number of levels (fv3gfs-util's QuantityHaloSpec)."""

    def __init__(self, dims, n_halo, nlev):
        self.dims = tuple(dims)
        self.n_points = int(n_halo)
        self.nlev = int(nlev)


def spec_for(grid_indexing, dims, n_halo=None):
    nlev = grid_indexing.npz + (1 if Z_INTERFACE_DIM in dims else 0)
    return HaloSpec(dims, grid_indexing.n_halo if n_halo is None else n_halo, nlev)


class _Updater:
    def __init__(self, comm, kind, specs):
        self._comm = comm
        self._kind = kind
        self._specs = specs

    def start(self, *quantity_lists):
        self._comm._run(self._kind, self._specs, quantity_lists)

    def wait(self):
        return None

    def update(self, *quantity_lists):
        self.start(*quantity_lists)


class DeviceCubedSphereCommunicator:
    """``get_scalar_halo_updater``, ``get_vector_halo_updater`` and
    ``synchronize_vector_interfaces`` for device tensors in kernel layout."""

    def __init__(self, grid_indexing):
        self._gi = grid_indexing

    @property
    def _ctx(self):
        if self._gi.context is None:
            raise RuntimeError("no device context on this grid (build a GridData first)")
        return self._gi.context

    def get_scalar_halo_updater(self, specs):
        for sp in specs:
            if (X_INTERFACE_DIM in sp.dims) != (Y_INTERFACE_DIM in sp.dims):
                raise NotImplementedError("scalar halo updates need the same staggering on x and y")
        return _Updater(self, "scalar", list(specs))

    def get_vector_halo_updater(self, specs_x, specs_y):
        return _Updater(self, "vector", (list(specs_x), list(specs_y)))

    def _run(self, kind, specs, quantity_lists):
        if kind == "scalar":
            (fields,) = quantity_lists
            for f, sp in zip(fields, specs):
                stagger = 0 if X_INTERFACE_DIM in sp.dims else 1
                _lib.call_ctx("fv3b_halo_update_scalar", self._ctx, f.data_ptr(), stagger, sp.n_points, sp.nlev,
                              stream_ptr())
        else:
            xs, ys = quantity_lists
            for x, y, sp in zip(xs, ys, specs[0]):
                grid = 1 if X_INTERFACE_DIM in sp.dims else 0  # C grid: x component on x interfaces
                _lib.call_ctx("fv3b_halo_update_vector", self._ctx, x.data_ptr(), y.data_ptr(), grid, sp.nlev,
                              stream_ptr())

    def synchronize_vector_interfaces(self, u, v):
        _lib.call_ctx("fv3b_synchronize_vector_interfaces", self._ctx, u.data_ptr(), v.data_ptr(), self._gi.npz,
                      stream_ptr())
