"""B200-native masstree: IndexinGPU's gpu_masstree hot path on sm_100a.

The product is libmt_b200.so (CUDA kernels behind the C ABI declared in
include/mt_masstree.h).  This package holds its Python host mirror
(GpuMasstree), the build step and the seeded workload generators.
"""
from .masstree import (FLAG_CONCURRENT, FLAG_UPDATE_IF_EXISTS, FLAG_USE_UPPER_KEY, REQ_ERASE, REQ_FIND, REQ_INSERT,
                       REQ_UPDATE, GpuMasstree, MasstreeError)

__all__ = ["GpuMasstree", "MasstreeError", "REQ_INSERT", "REQ_ERASE", "REQ_FIND", "REQ_UPDATE", "FLAG_CONCURRENT",
           "FLAG_UPDATE_IF_EXISTS", "FLAG_USE_UPPER_KEY"]
