"""cosmosphere_b200: a B200-native (sm_100a) drop-in for cosmoSPHere's SPH density /
smoothing-length / force path.

The product is the C-ABI shared library ``lib/libcosmoSPHere.so`` (M4 cubic kernel) and
``lib/libcosmoSPHere_quintic.so`` (M6 quintic), declared in ``include/cosmosphere.h``.
This package is a thin ctypes binding of it (``capi``) plus the seeded synthetic input
generators (``inputs``).  There is no CPU fallback: importing ``capi`` without the built
library raises.
"""
from . import capi, inputs  # noqa: F401

__all__ = ["capi", "inputs"]
