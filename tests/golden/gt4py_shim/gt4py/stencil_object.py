from .gtscript import StencilObject  # noqa: F401
