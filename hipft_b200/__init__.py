"""hipft_b200 -- B200 (sm_100a) flux-transport step of HipFT behind a C ABI.

The CUDA library (libhipft_gpu.so, include/hipft_gpu.h) holds the kernels
and the driver; :mod:`hipft_b200.gpu` is its ctypes binding.
"""
from .gpu import HipftGPU, HipftError, h5_read, h5_write, lib, run, run_field  # noqa: F401

__all__ = ["HipftGPU", "HipftError", "h5_read", "h5_write", "lib", "run", "run_field"]
