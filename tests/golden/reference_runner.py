"""Run the reference's own stencil classes on the CPU (this container only).

The reference (fv3core, pure gtscript) needs gt4py v36 and fv3gfs-util,
neither of which is installed.  ``gt4py_shim/`` holds a minimal gtscript
interpreter with gt4py-numpy-backend semantics and the few fv3gfs.util names
the hot path imports; with them the reference modules import unchanged from
the checkout named by the ``FV3CORE_REFERENCE`` environment variable (the
directory that holds the ``fv3core`` package) and their stencil classes
execute.  Results are
written as golden fixtures by ``make_golden.py``; nothing here is used on
the GPU box or by the product.
"""
import os
import sys
import threading
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def reference_root():
    """The reference checkout, from ``FV3CORE_REFERENCE`` (required)."""
    root = os.environ.get("FV3CORE_REFERENCE")
    if not root:
        raise RuntimeError("set FV3CORE_REFERENCE to the reference checkout (the directory holding fv3core/)")
    if not os.path.isdir(os.path.join(root, "fv3core")):
        raise RuntimeError(f"FV3CORE_REFERENCE={root!r} holds no fv3core package")
    return root


def import_reference():
    REFERENCE = reference_root()
    if HERE + "/gt4py_shim" not in sys.path:
        sys.path.insert(0, os.path.join(HERE, "gt4py_shim"))
    if REFERENCE not in sys.path:
        sys.path.insert(0, REFERENCE)
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    if not hasattr(np, "float_"):
        np.float_ = np.float64  # removed in numpy 2; the reference's typing.py uses it
    import fv3core  # noqa: F401
    import fv3core.utils.global_config as gc

    gc.set_backend("numpy")
    gc.set_validate_args(False)
    return fv3core


def storage(arr, origin=(3, 3, 0)):
    from gt4py.storage import Storage

    st = np.array(arr, dtype=np.float64, copy=True).view(Storage)
    st.default_origin = origin
    return st


class _LegacyGrid:
    """Stand-in for the reference's global ``spec.grid`` (hashable by identity,
    as fv3core caches axis offsets per grid object)."""


class TileReference:
    """Reference objects (grid data, stencil factory, legacy ``spec.grid``)
    for one tile of a ``CubedSphereGrid``."""

    def __init__(self, grid, tile, nz):
        import_reference()
        import fv3core._config as spec
        from fv3core.utils.grid import (
            AngleGridData,
            ContravariantGridData,
            DampingCoefficients,
            GridData,
            HorizontalGridData,
            VerticalGridData,
        )
        from fv3core.utils.stencil import GridIndexing, StencilConfig, StencilFactory

        self.grid, self.tile, self.nz = grid, tile, nz
        n, h = grid.n, grid.halo
        g = grid
        t = tile

        def ij(name):
            return storage(getattr(g, name)[t], origin=(h, h))

        horizontal = HorizontalGridData(
            area=ij("area"),
            area_64=ij("area"),
            rarea=ij("rarea"),
            rarea_c=ij("rarea_c"),
            dx=ij("dx"),
            dy=ij("dy"),
            dxc=ij("dxc"),
            dyc=ij("dyc"),
            dxa=ij("dxa"),
            dya=ij("dya"),
            rdx=ij("rdx"),
            rdy=ij("rdy"),
            rdxc=ij("rdxc"),
            rdyc=ij("rdyc"),
            rdxa=ij("rdxa"),
            rdya=ij("rdya"),
        )
        contravariant = ContravariantGridData(
            ij("cosa"),
            ij("cosa_u"),
            ij("cosa_v"),
            ij("cosa_s"),
            ij("sina_u"),
            ij("sina_v"),
            ij("rsina"),
            ij("rsin_u"),
            ij("rsin_v"),
            ij("rsin2"),
        )
        angle = AngleGridData(
            ij("sin_sg1"),
            ij("sin_sg2"),
            ij("sin_sg3"),
            ij("sin_sg4"),
            ij("cos_sg1"),
            ij("cos_sg2"),
            ij("cos_sg3"),
            ij("cos_sg4"),
        )
        self.grid_data = GridData(horizontal, VerticalGridData(), contravariant, angle)
        self.damping_coefficients = DampingCoefficients(
            del6_u=ij("del6_u"), del6_v=ij("del6_v"), da_min=g.da_min, da_min_c=g.da_min_c
        )
        m = n + 2 * h + 1
        legacy = _LegacyGrid()
        legacy.fC = ij("fC")
        legacy.f0 = ij("f0")
        legacy.npz = nz
        legacy.nested = False
        legacy.grid_type = 0
        legacy.stretched_grid = False
        legacy.rank = t
        legacy.agrid1 = ij("agrid1")
        legacy.agrid2 = ij("agrid2")
        legacy.bgrid1 = ij("bgrid1")
        legacy.bgrid2 = ij("bgrid2")
        legacy.divg_u = ij("divg_u")
        legacy.divg_v = ij("divg_v")
        # edge factors: west/east as IJ fields singleton in i, south/north as I fields
        ew = np.zeros((1, m))
        ew[0, h : h + n + 1] = g.edge_w[t]
        ee = np.zeros((1, m))
        ee[0, h : h + n + 1] = g.edge_e[t]
        es = np.zeros(m)
        es[h : h + n + 1] = g.edge_s[t]
        en = np.zeros(m)
        en[h : h + n + 1] = g.edge_n[t]
        legacy.edge_w = storage(ew, origin=(0, 0))
        legacy.edge_e = storage(ee, origin=(0, 0))
        legacy.edge_s = storage(es, origin=(0,))
        legacy.edge_n = storage(en, origin=(0,))
        spec.grid = legacy
        self.legacy = legacy
        self.spec = spec
        self.grid_indexing = GridIndexing((n, n, nz), h, True, True, True, True)
        legacy.axis_offsets = self.grid_indexing.axis_offsets
        self.stencil_factory = StencilFactory(StencilConfig("numpy", False, False), self.grid_indexing)

    def activate(self):
        """Make this tile's legacy grid the global one (constructors read it)."""
        self.spec.grid = self.legacy

    def add_tracer_grid(self):
        """The legacy-grid members TracerAdvection reads
        (tracer_2d_1l.py:143-200): metric terms, quantity_wrap and
        get_halo_update_spec."""
        import fv3gfs.util as fu

        g, t, h, nz = self.grid, self.tile, self.grid.halo, self.nz
        legacy = self.legacy
        for name in ("dxa", "dya", "dx", "dy", "sin_sg1", "sin_sg2", "sin_sg3", "sin_sg4", "rarea"):
            setattr(legacy, name, storage(getattr(g, name)[t], origin=(h, h)))
        sizer = fu.SubtileGridSizer(g.n, g.n, nz, h)
        gi = self.grid_indexing

        def quantity_wrap(data, dims=(fu.X_DIM, fu.Y_DIM, fu.Z_DIM), units="Unknown"):
            return fu.Quantity(data, dims=dims, units=units, origin=sizer.get_origin(dims),
                               extent=sizer.get_extent(dims))

        def get_halo_update_spec(shape, origin, halo_points, dims=(fu.X_DIM, fu.Y_DIM, fu.Z_DIM)):
            return gi.get_quantity_halo_spec(shape, origin, dims=list(dims), n_halo=halo_points)

        legacy.quantity_wrap = quantity_wrap
        legacy.get_halo_update_spec = get_halo_update_spec
        for name in ("a11", "a12", "a21", "a22"):
            setattr(legacy, name, storage(getattr(g, name)[t], origin=(h, h)))


# ---------------------------------------------------------------------------
# Six tiles in lock step: a fake communicator whose halo updaters exchange
# between threads, in the manner of the reference's mock-parallel tests
# (tests/savepoint/conftest.py:516-535).
class _Exchange:
    def __init__(self):
        self.lock = threading.Condition()
        self.posts = {}

    def post(self, key, tile, payload):
        with self.lock:
            self.posts.setdefault(key, {})[tile] = payload
            self.lock.notify_all()

    def collect(self, key, timeout=600.0):
        with self.lock:
            ok = self.lock.wait_for(lambda: len(self.posts.get(key, {})) == 6, timeout=timeout)
            if not ok:
                raise RuntimeError(f"halo exchange {key} timed out")
            return self.posts[key]


class _HaloUpdater:
    def __init__(self, comm, kind, specs):
        self.comm = comm
        self.kind = kind
        self.specs = specs
        self.gen = 0
        self._pending = None

    def start(self, *quantity_lists):
        comm = self.comm
        key = (self.kind, comm.uid_of(self), self.gen)
        self.gen += 1
        snap = [[np.array(q.data, copy=True) for q in ql] for ql in quantity_lists]
        comm.exchange.post(key, comm.tile, snap)
        self._pending = (key, quantity_lists)

    def wait(self):
        key, quantity_lists = self._pending
        posts = self.comm.exchange.collect(key)
        self.comm.fill(self.kind, self.specs, quantity_lists, posts)
        self._pending = None

    def update(self, *quantity_lists):
        self.start(*quantity_lists)
        self.wait()


class ThreadComm:
    """Communicator for one tile; all six share ``exchange``."""

    def __init__(self, tile, n, h, exchange):
        self.tile = tile
        self.n, self.h = n, h
        self.exchange = exchange
        self._uids = {}
        self._vector_updaters = {}
        self.sync_gen = 0

    def uid_of(self, updater):
        if id(updater) not in self._uids:
            self._uids[id(updater)] = len(self._uids)
        return self._uids[id(updater)]

    def get_scalar_halo_updater(self, specs):
        return _HaloUpdater(self, "scalar", specs)

    def get_vector_halo_updater(self, specs_x, specs_y):
        return _HaloUpdater(self, "vector", (specs_x, specs_y))

    def fill(self, kind, specs, quantity_lists, posts):
        from fv3core_b200 import halo_map as hm

        n, h, t = self.n, self.h, self.tile
        if kind == "scalar":
            (qlist,) = quantity_lists
            for qi, (q, spec) in enumerate(zip(qlist, specs)):
                sx = 0 if "x_interface" in q.dims else 1
                sy = 0 if "y_interface" in q.dims else 1
                nh = spec.n_points
                nk = spec.extent[-1]
                table = hm.scalar_table(n, h, sx, sy, nh)
                rows = table[table[:, 0] == t]
                for r in rows:
                    src = posts[r[3]][0][qi]
                    q.data[r[1], r[2], :nk] = src[r[4], r[5], :nk]
        else:
            qx_list, qy_list = quantity_lists
            for qi in range(len(qx_list)):
                qx, qy = qx_list[qi], qy_list[qi]
                stx = (0 if "x_interface" in qx.dims else 1, 0 if "y_interface" in qx.dims else 1)
                sty = (0 if "x_interface" in qy.dims else 1, 0 if "y_interface" in qy.dims else 1)
                nh = specs[0][qi].n_points
                nk = specs[0][qi].extent[-1]
                tables = hm.vector_tables(n, h, stx, sty, nh)
                for dst, table in zip((qx, qy), tables):
                    rows = table[table[:, 0] == t]
                    for r in rows:
                        src = posts[r[3]][r[6]][qi]
                        dst.data[r[1], r[2], :nk] = r[7] * src[r[4], r[5], :nk]

    def vector_halo_update(self, u_q, v_q, n_points):
        """CubedSphereCommunicator.vector_halo_update: one blocking vector
        exchange (as CubedToLatLon calls it)."""
        from types import SimpleNamespace

        nk = u_q.extent[-1]
        key = ("vector_halo_update", n_points, nk)
        if key not in self._vector_updaters:  # one updater per shape: keys stay unique
            spec = SimpleNamespace(n_points=n_points, extent=(0, 0, nk))
            self._vector_updaters[key] = _HaloUpdater(self, "vector", ([spec], [spec]))
        self._vector_updaters[key].update([u_q], [v_q])

    def synchronize_vector_interfaces(self, u_q, v_q):
        from fv3core_b200 import halo_map as hm

        key = ("sync", self.sync_gen)
        self.sync_gen += 1
        self.exchange.post(key, self.tile, [np.array(u_q.data, copy=True), np.array(v_q.data, copy=True)])
        posts = self.exchange.collect(key)
        table = hm.interface_sync_tables(self.n, self.h)
        nk = u_q.extent[-1]
        for r in table[table[:, 0] == self.tile]:
            dst = (u_q, v_q)[r[1]]
            src = posts[r[4]][r[5]]
            dst.data[r[2], r[3], :nk] = r[8] * src[r[6], r[7], :nk]
