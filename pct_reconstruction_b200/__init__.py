"""B200-native proton-CT reconstruction engine (drop-in for the MLP + DROP path of
BlakeSchultze/pCT_Reconstruction).

The compute lives in libpct_b200.so (hand-written sm_100a CUDA behind the C ABI of
include/pct_api.h); this package is the Python host side: configuration with the reference's
parameter names, a context wrapper with the reference's stage names, and synthetic phantoms.
"""
from ._abi import LIB_PATH, load_library  # noqa: F401
from .engine import Batch, Config, Context, PCTError  # noqa: F401

__all__ = ["Batch", "Config", "Context", "PCTError", "load_library", "LIB_PATH"]
