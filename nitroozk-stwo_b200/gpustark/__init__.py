"""gpustark: B200-native Circle-STARK proving backend (Python host binding).

The compute path is libgpustark.so (hand-written sm_100a CUDA behind the C ABI
in include/gpustark.h). This package only binds it; it has no CPU fallback.
"""
from ._lib import GpuStarkError, LIB_PATH, declared_symbols, lib  # noqa: F401

__all__ = ["GpuStarkError", "LIB_PATH", "declared_symbols", "lib"]
