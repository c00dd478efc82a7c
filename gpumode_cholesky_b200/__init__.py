"""gpumode_cholesky_b200 -- batched Cholesky (potrf) for NVIDIA B200 (sm_100a).

Drop-in for the GPU MODE ``cholesky`` entry point ``custom_kernel(A) -> L``
(binga/gpumode_cholesky, submission.py:4101-4268): hand-written CUDA kernels
behind a C ABI (``include/b200_potrf.h``), called from Python through ctypes.
"""

from ._lib import LaunchTrace, PotrfError
from .autograd import CholeskyFunction, cholesky_differentiable, potrf_backward
from .gp import gp_nll, trsv
from .potrf import cholesky, cholesky_checked, cholesky_host, custom_kernel

__all__ = [
    "CholeskyFunction",
    "LaunchTrace",
    "PotrfError",
    "cholesky",
    "cholesky_checked",
    "cholesky_host",
    "cholesky_differentiable",
    "custom_kernel",
    "gp_nll",
    "potrf_backward",
    "trsv",
]
