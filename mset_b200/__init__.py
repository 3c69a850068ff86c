"""mset_b200 -- B200-native (sm_100a) multislice forward/adjoint hot path of
MSET (multislice electron tomography from 4D-STEM tilt series).

The compute path is libmset_b200.so (hand-written CUDA kernels behind the C
ABI in include/mset_b200.h); this package is its host-side mirror of the
reference's MEX interface (:mod:`mset_b200.session`), the batched method
(:mod:`mset_b200.batch`), host physics set-up and the synthetic data
generator.
"""
from ._lib import (MSET_ADJOINT_EXACT, MSET_ADJOINT_REF, MSET_E_ARG, MSET_E_CUDA, MSET_E_NOMEM, MSET_E_STATE,
                   MSET_E_UNSUPPORTED, MSET_MODE_MSET, MSET_MODE_SSET, MsetError, LIB_PATH, load)
from .session import Session, mset_cuda_kernel, clear

__all__ = ["Session", "mset_cuda_kernel", "clear", "MsetError", "load", "LIB_PATH",
           "MSET_MODE_MSET", "MSET_MODE_SSET", "MSET_ADJOINT_REF", "MSET_ADJOINT_EXACT", "MSET_E_ARG",
           "MSET_E_UNSUPPORTED", "MSET_E_CUDA", "MSET_E_STATE", "MSET_E_NOMEM"]
