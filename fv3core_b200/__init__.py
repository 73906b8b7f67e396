"""B200-native acoustic substep of the FV3 nonhydrostatic dynamical core.

The package keeps the reference's (fv3core) stencil-class API for the
acoustic substep and runs every stencil as a hand-written sm_100a CUDA
kernel through the C-ABI library ``libfv3core_b200.so``.
"""
__version__ = "0.1.0"
