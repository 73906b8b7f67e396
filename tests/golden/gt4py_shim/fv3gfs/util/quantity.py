from . import Quantity  # noqa: F401
