"""shtools_b200 -- B200-native real spherical harmonic transforms.

GPU implementation of the SHTOOLS transforms MakeGridDH / SHExpandDH and
MakeGridGLQ / SHExpandGLQ (every norm, csphase, sampling, lmax_calc and
extend option), their complex counterparts MakeGridDHC / SHExpandDHC /
MakeGridGLQC / SHExpandGLQC, the quadrature routines PreGLQ / SHGLQ / DHaj, and their
adjoints for autograd.  The arithmetic runs in hand-written sm_100a kernels
of libshtcuda (shtools_b200/csrc, C ABI in include/shtcuda.h); PyTorch
provides device memory and streams.

    import shtools_b200 as sht
    grid = sht.MakeGridDH(cilm_cuda, sampling=2)      # torch, differentiable
    cilm = sht.SHExpandDH(grid, sampling=2)

    from shtools_b200 import backend
    backend.register()                                # pyshtools 'cuda'
"""
from .transforms import (MakeGridDH, SHExpandDH, MakeGridGLQ, SHExpandGLQ,
                         MakeGridDHC, SHExpandDHC, MakeGridGLQC, SHExpandGLQC,
                         MakeGradientDH, MakeGravGridDH, NormalGravity, SHMultiply,
                         PreGLQ, SHGLQ, DHaj, Plan, get_plan,
                         clear_plan_cache, mixed_status, GRID_DH, GRID_GLQ)
from ._lib import SHTCudaError

__all__ = ["MakeGridDH", "SHExpandDH", "MakeGridGLQ", "SHExpandGLQ",
           "MakeGridDHC", "SHExpandDHC", "MakeGridGLQC", "SHExpandGLQC",
           "MakeGradientDH", "MakeGravGridDH", "NormalGravity", "SHMultiply", "PreGLQ",
           "SHGLQ", "DHaj", "Plan", "get_plan", "clear_plan_cache", "mixed_status", "GRID_DH",
           "GRID_GLQ", "SHTCudaError"]
