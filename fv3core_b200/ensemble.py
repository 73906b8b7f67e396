"""Ensembles of independent cubed-sphere states advanced together.

The members of one resolution form a ``MemberGroup``: their states live in
one batched context (``GridData(members=M)``, fv3b_ctx_create_batched), so
every kernel of an AcousticDynamics call advances all of them in one launch
(the grid's tile dimension covers 6 x M tile slots; halo updates stay
within a member).  An ensemble at mixed resolutions is one group per
resolution, and a step is one AcousticDynamics call per group.  ``capture``
records a whole ensemble step in one CUDA graph.  ``Member`` (one context
per member, one call per member) is the unbatched form, kept for
comparison.
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


class MemberGroup:
    """Members of one resolution (n, npz), one seed each, in one batched
    context: every kernel of a step covers all of them."""

    def __init__(self, n, npz, seeds, precision="f64", n_split=6, mdt=225.0, noise=1.0e-3, grid=None):
        self.n, self.npz, self.seeds = n, npz, list(seeds)
        grid = CubedSphereGrid(n, 3) if grid is None else grid
        states = [baroclinic_state(grid, npz, seed=s, noise=noise) for s in self.seeds]
        st0 = states[0]
        self.grid_data = GridData(grid, npz, precision=precision, members=len(self.seeds))
        gi = self.grid_data.grid_indexing
        state = types.SimpleNamespace()
        for name in _lib.DYCORE_FIELDS:
            parts = [st[name] if name in st else np.zeros(st["phis"].shape if name == "wsd" else st["delp"].shape)
                     for st in states]
            setattr(state, name, to_device(np.concatenate(parts, axis=0), dtype=gi.dtype))
        state.mdt, state.n_map, state.akap = mdt, 1, 287.05 / 1004.6
        state.ptop, state.ks = st0["ptop"], st0["ks"]
        self.state = state
        self.dynamics = AcousticDynamics(
            DeviceCubedSphereCommunicator(gi), StencilFactory(StencilConfig(), gi), self.grid_data, self.grid_data,
            0, False, False, baroclinic_acoustic_config(n_split=n_split), st0["ak"], st0["bk"], st0["pfull"],
            state.phis,
        )
        self.cell_levels = len(self.seeds) * 6 * n * n * npz
        self._initial = None

    def member_field(self, name, m):
        """Member m's tiles of a state field (a view)."""
        return getattr(self.state, name)[6 * m:6 * m + 6]

    keep_initial = Member.keep_initial
    reset = Member.reset
    step = Member.step
    close = Member.close


class Ensemble:
    """members: iterable of (n, npz, seed).  ``batched`` (default): the
    members of each resolution share one batched context (MemberGroup), in
    the order in which their resolutions first appear; otherwise one context
    per member."""

    def __init__(self, members, precision="f64", n_split=6, batched=True):
        self.n_split = n_split
        grids = {}
        members = list(members)
        for n, npz, seed in members:
            if n not in grids:
                grids[n] = CubedSphereGrid(n, 3)
        self.members = []
        if batched:
            order = []
            seeds = {}
            for n, npz, seed in members:
                if (n, npz) not in seeds:
                    order.append((n, npz))
                    seeds[(n, npz)] = []
                seeds[(n, npz)].append(seed)
            for n, npz in order:
                self.members.append(MemberGroup(n, npz, seeds[(n, npz)], precision, n_split, grid=grids[n]))
        else:
            for n, npz, seed in members:
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
