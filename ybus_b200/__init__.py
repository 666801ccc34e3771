"""ybus_b200: a B200-native factor-once / solve-many engine for ybus's GPU path.

A sparse Cholesky or LU factor, made once on the host in FP64, is uploaded and then solved for
large blocks of right-hand sides by hand-written sm_100a kernels, behind a C ABI that mirrors
ybus_cuda's API (include/ybgpu.h). Python mirrors that API on top of the C ABI.
"""
from . import grids, host
from ._lib import YbError
from .gpu import (FP32, FP64, ColumnMax, CudaError, Gpu, GpuBlock, GpuFactor, GpuOperator, Pair, PairUpdate,
                  ShapeMismatch, Timings, solve_batch_complex)

__all__ = ["grids", "host", "Gpu", "GpuFactor", "GpuBlock", "GpuOperator", "Pair", "PairUpdate", "ColumnMax", "Timings",
           "CudaError", "ShapeMismatch", "YbError", "FP64", "FP32", "solve_batch_complex"]
