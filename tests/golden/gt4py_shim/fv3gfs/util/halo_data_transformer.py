import dataclasses
from typing import Any, Tuple


@dataclasses.dataclass
class QuantityHaloSpec:
    n_points: int
    strides: Tuple[int, ...]
    itemsize: int
    shape: Tuple[int, ...]
    origin: Tuple[int, ...]
    extent: Tuple[int, ...]
    dims: Tuple[str, ...]
    numpy_module: Any
    dtype: Any
