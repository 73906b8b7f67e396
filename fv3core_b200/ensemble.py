"""Ensembles of independent cubed-sphere states advanced together.

Each member is a full AcousticDynamics problem (its own grid, context and
state) at its own resolution.  ``step`` enqueues one AcousticDynamics call
(n_split acoustic substeps) per member, eagerly; ``capture`` records the
whole ensemble step, every member's launches, in one CUDA graph, so a step
costs one graph launch instead of ~1000 kernel launches per member.
"""
import types

import numpy as np
import torch

from . import _lib
from .config import baroclinic_acoustic_config
from .grid import CubedSphereGrid
from .grid_data import GridData
from .halo import DeviceCubedSphereCommunicator
from .initial_state import baroclinic_state
from .stencil import StencilConfig, StencilFactory
from .stencils.dyn_core import AcousticDynamics
from .storage import to_device


class Member:
    def __init__(self, n, npz, seed, precision="f64", n_split=6, mdt=225.0, noise=1.0e-3, grid=None):
        self.n, self.npz, self.seed = n, npz, seed
        grid = CubedSphereGrid(n, 3) if grid is None else grid
        st = baroclinic_state(grid, npz, seed=seed, noise=noise)
        self.grid_data = GridData(grid, npz, precision=precision)
        gi = self.grid_data.grid_indexing
        state = types.SimpleNamespace()
        for name in _lib.DYCORE_FIELDS:
            a = st[name] if name in st else np.zeros(st["phis"].shape if name == "wsd" else st["delp"].shape)
            setattr(state, name, to_device(a, dtype=gi.dtype))
        state.mdt, state.n_map, state.akap = mdt, 1, 287.05 / 1004.6
        state.ptop, state.ks = st["ptop"], st["ks"]
        self.state = state
        self.dynamics = AcousticDynamics(
            DeviceCubedSphereCommunicator(gi), StencilFactory(StencilConfig(), gi), self.grid_data, self.grid_data,
            0, False, False, baroclinic_acoustic_config(n_split=n_split), st["ak"], st["bk"], st["pfull"], state.phis,
        )
        self.cell_levels = 6 * n * n * npz
        self._initial = None

    def keep_initial(self):
        """Keep a device copy of the current state for ``reset``."""
        self._initial = {k: getattr(self.state, k).clone() for k in _lib.DYCORE_FIELDS}

    def reset(self):
        """Copy the kept state back (device to device, capturable)."""
        for k, t in self._initial.items():
            getattr(self.state, k).copy_(t)

    def step(self, reset=False):
        if reset:
            self.reset()
        self.dynamics(self.state)

    def close(self):
        self.grid_data.close()


class Ensemble:
    """members: iterable of (n, npz, seed)."""

    def __init__(self, members, precision="f64", n_split=6):
        self.n_split = n_split
        grids = {}
        self.members = []
        for n, npz, seed in members:
            if n not in grids:
                grids[n] = CubedSphereGrid(n, 3)
            self.members.append(Member(n, npz, seed, precision, n_split, grid=grids[n]))

    @property
    def cell_levels(self):
        return sum(m.cell_levels for m in self.members)

    def keep_initial(self):
        for m in self.members:
            m.keep_initial()

    def step(self, reset=False):
        """One AcousticDynamics call per member; with ``reset`` every member
        first returns to its kept state (``keep_initial``)."""
        for m in self.members:
            m.step(reset)

    def capture(self, reset=False):
        """One CUDA graph of a whole ensemble step.  Every member must have
        stepped eagerly once (the per-level Rayleigh factors are uploaded by
        the first call); replaying the graph advances all members."""
        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph):
            self.step(reset)
        return graph

    def close(self):
        for m in self.members:
            m.close()
