"""``AcousticDynamics`` — reference ``fv3core/stencils/dyn_core.py:210-761``.

The whole substep loop runs in the native library (``fv3b_acoustics``): one
call enqueues every stage and halo gather of the n_split acoustic substeps
on the current CUDA stream.
"""
import ctypes

import numpy as np

from .. import _lib
from ..storage import check_field, stream_ptr
from ._common import host_column

TEMPORARIES = ("gz", "zh", "pkc", "pk3", "ut", "vt", "divgd", "heat_source", "crx", "cry", "xfx", "yfx", "delpc",
               "ptc", "ws3", "zs", "dp_ref")


class AcousticDynamics:
    """Fortran name dyn_core: the Lagrangian acoustic dynamics of Lin 2004
    for all six tiles.

    ``comm`` is accepted for interface compatibility (the halo exchanges are
    on-device gathers); ``grid_data`` must be a ``fv3core_b200.grid_data.GridData``.
    ``ak``, ``bk``, ``pfull`` are K fields (host arrays or tensors) and
    ``phis`` a 2-D device field.
    """

    def __init__(self, comm, stencil_factory, grid_data, damping_coefficients, grid_type, nested, stretched_grid,
                 config, ak, bk, pfull, phis):
        if nested or stretched_grid:
            raise NotImplementedError("nested and stretched grids are not supported")
        if config.d_ext != 0:
            raise AssertionError("d_ext != 0 is not implemented")
        if config.beta != 0:
            raise AssertionError("beta != 0 is not implemented")
        if config.use_logp:
            raise AssertionError("use_logp=True is not implemented")
        if config.riemann.a_imp <= 0.999:
            raise NotImplementedError("a_imp <= 0.999 is not implemented")
        self.comm = comm
        self.config = config
        self.grid_data = grid_data
        self._gi = stencil_factory.grid_indexing
        gi = self._gi
        self._ctx = grid_data.ctx
        npz = gi.npz
        c = _lib.AcousticConfig()
        c.tau, c.delt_max, c.rf_cutoff, c.p_fac = config.tau, config.delt_max, config.rf_cutoff, config.p_fac
        c.k_split, c.n_split = config.k_split, config.n_split
        c.rf_fast, c.breed_vortex_inline = int(config.rf_fast), int(config.breed_vortex_inline)
        c.use_old_omega = int(config.use_old_omega)
        self._config = c
        d = _lib.DswConfig()
        for name, _ in _lib.DswConfig._fields_:
            setattr(d, name, type(getattr(d, name))(getattr(config.d_grid_shallow_water, name)))
        self._dsw = d
        self._ak = host_column(ak, npz + 1, "ak")
        self._bk = host_column(bk, npz + 1, "bk")
        self._pfull = host_column(pfull, npz, "pfull")
        _lib.call_ctx(
            "fv3b_acoustics_setup", self._ctx, ctypes.addressof(c), ctypes.addressof(d), self._ak.ctypes.data,
            self._bk.ctypes.data, self._pfull.ctypes.data, check_field(phis, gi, "2d", "phis"),
        )
        self._state = _lib.DycoreState()

    def temporary(self, name):
        """One of the substep temporaries as a torch tensor sharing the
        library's memory (3-D kernel layout; ws3 and zs 2-D; dp_ref 1-D)."""
        import torch

        if name not in TEMPORARIES:
            raise KeyError(name)
        ptr = _lib.lib(self._gi.precision).fv3b_acoustics_temporary(self._ctx, name.encode())
        m, _, nk = self._gi.max_shape
        nt = self._gi.ntiles
        shape = {"ws3": (nt, m, m), "zs": (nt, m, m), "dp_ref": (nk,)}.get(name, (nt, nk, m, m))

        class _View:
            __cuda_array_interface__ = {"shape": shape, "typestr": "<f4" if self._gi.precision == "f32" else "<f8",
                                        "data": (ptr, False), "version": 3,
                                        "strides": None}

        return torch.as_tensor(_View(), device="cuda")

    def __call__(self, state):
        gi = self._gi
        s = self._state
        for name in _lib.DYCORE_FIELDS:
            kind = "2d" if name in ("phis", "wsd") else "3d"
            setattr(s, name, check_field(getattr(state, name), gi, kind, name))
        s.mdt = float(state.mdt)
        s.akap = float(getattr(state, "akap", 0.0))
        s.ptop = float(state.ptop)
        s.n_map = int(state.n_map)
        s.ks = int(getattr(state, "ks", 0))
        _lib.call_ctx("fv3b_acoustics", self._ctx, ctypes.addressof(s), stream_ptr())

    def capture(self, state):
        """Record one call on ``state`` in a CUDA graph and return it;
        ``graph.replay()`` then advances the same tensors.  Make one eager
        call first: it uploads the per-level Rayleigh factors, which a
        capture cannot do."""
        import torch

        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph):
            self(state)
        return graph
