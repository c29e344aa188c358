"""lambda_vm_b200 — B200-native (sm_100a) Goldilocks STARK proving backend.

The CUDA kernels and the C ABI live in csrc/ and include/starkgpu.h
(libstarkgpu.so); `math_cuda` mirrors the reference's math-cuda API on top of
that ABI. There is no CPU fallback: importing the compute modules requires the
built library.
"""
from . import native  # noqa: F401

__all__ = ["native", "device", "math_cuda"]
