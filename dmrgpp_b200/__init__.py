"""dmrgpp_b200: B200-native superblock H*psi engine for DMRG++.

The compute path is the CUDA library ``_lib/libdmrgpp_kron.so`` (sources in
``csrc/``, C ABI in ``include/dmrgpp_kron.h``).  Python here is a thin
binding used by tests and benchmarks; there is no CPU fallback.
"""
from ._capi import DmrgppError, FP64, SPLIT_BF16, TF32X3  # noqa: F401

__all__ = ["DmrgppError", "FP64", "SPLIT_BF16", "TF32X3"]
