"""vmachine_b200: B200-native walker engine for VMaChine's Metropolis / local-energy path.

The engine is libvmc_b200.so (hand-written sm_100a CUDA behind the C ABI in
include/vmc_b200.h); this package is its Python binding.
"""
from .engine import (EXPORTS, LIB_PATH, Averages, Batch, Engine, Info, Options, Sums,  # noqa: F401
                     VmcError, block_series, library, measure_fma_peak)

__all__ = ["Engine", "Batch", "VmcError", "library", "LIB_PATH", "EXPORTS", "Averages", "Sums", "Info",
           "Options", "measure_fma_peak", "block_series"]
