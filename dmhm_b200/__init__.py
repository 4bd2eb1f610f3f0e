"""dmhm_b200: B200 (sm_100a) H-matrix engine.

A from-scratch GPU implementation of the hot paths of YingzhouLi/dmhm's
serial HMat2d / HMat3d: H-matrix x vector / dense products, the H*H product
with randomized low-rank compression, and Schulz inversion.  The numeric work
runs in hand-written CUDA kernels behind the C ABI of
``include/dmhm_b200.h`` (``libdmhm_b200.so``); this package is the thin
Python mirror of the reference's C++ API.
"""
from ._lib import HMError, LIB_PATH, lib
from .hmat import (Context, DistHMat2d, DistHMat3d, EstimateTwoNorm, Finalize, HMat2d, HMat3d,
                   Initialize, Teams,
                   Oversample, SetOversample, SetCompressionTolerance, CompressionTolerance,
                   RankModel, Sparse, natural_to_hierarchical_map)
from . import operators

__all__ = ["Context", "DistHMat2d", "DistHMat3d", "EstimateTwoNorm", "Finalize", "HMError",
           "HMat2d", "HMat3d", "Initialize", "Teams",
           "LIB_PATH", "Oversample", "SetOversample", "SetCompressionTolerance",
           "CompressionTolerance", "RankModel", "Sparse", "lib",
           "natural_to_hierarchical_map", "operators"]
