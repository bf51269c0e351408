"""nido_b200: a B200-native (sm_100a) Louvain community-detection engine with
the surface of sg0/nido.

The engine is libnido_b200.so (C ABI, include/nido_b200.h) built from
nido_b200/csrc; this package binds it for Python callers.  Importing the
package does not load the library; `nido_b200.capi.lib()` does, and raises if
it has not been built.
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
