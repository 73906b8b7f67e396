"""Minimal stand-in for the gt4py package (v36 API subset) used only by the
golden-fixture generator to run the reference's stencils on the CPU."""
from . import definitions, gtscript, storage  # noqa: F401
from .gtscript import StencilObject  # noqa: F401

__version__ = "0.0.0-shim"
