"""B200-native density-matrix step for PTB (submatrix method and purification).

The compute path is libptbgpu.so (CUDA for sm_100a, C-ABI in include/ptbgpu.h);
this package holds its host-side mirror of the reference interface.
"""
from .api import (OK, PREC_FP64, PREC_MIXED, PREC_MIXED_NOREFINE, Context, Options, PtbGpuError, Stats,
                  band_structure, get_nel, library_path, load_library, npacked)
from .settings import PurificationSettings

__all__ = ["Context", "Options", "Stats", "PtbGpuError", "PurificationSettings", "load_library", "library_path",
           "npacked", "get_nel", "band_structure", "PREC_FP64", "PREC_MIXED", "PREC_MIXED_NOREFINE", "OK"]
