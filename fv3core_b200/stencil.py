"""``StencilFactory`` / ``GridIndexing`` with the reference's names
(fv3core/utils/stencil.py:645-728): the object every stencil class takes."""
from .storage import GridIndexing  # noqa: F401


class StencilConfig:
    def __init__(self, backend="cuda-sm100a", rebuild=False, validate_args=True):
        self.backend = backend
        self.rebuild = rebuild
        self.validate_args = validate_args


class StencilFactory:
    def __init__(self, config, grid_indexing):
        self.config = config
        self.grid_indexing = grid_indexing
