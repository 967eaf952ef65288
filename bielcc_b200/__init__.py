"""bielcc_b200 — B200 (sm_100a) implementation of BIELcc's Stratton-Chu hot path.

The compute lives in libbielcc_gpu.so (CUDA kernels + C ABI, include/bielcc_gpu.h);
this package loads it lazily (bielcc_b200.gpu) and mirrors the reference's
operator interface for Python callers.
"""
__all__ = ["abi", "workloads"]
