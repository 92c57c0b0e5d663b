"""B200-native sparse iterative-solve path with the reference's interface.

Submodules:
  matrix        Csr / Ell / Sellp and the CudaExecutor (SpMV, conversions)
  solver        Cg / Bicgstab / Gmres / Ir factories over the fused solvers
  batch         batched BiCGStab on ragged batch Ell with its autotuner
  autograd      differentiable sparse solve (adjoint CG + SDDMM)
  mtx_io        MatrixMarket and binary matrix I/O (host code)
  stencils      seeded synthetic matrices of the benchmark workloads
  build         nvcc build of libginkgo_b200.so (sm_100a)

The CUDA library is loaded on first use; there is no CPU fallback.
"""
from ._lib import GinkgoError, declared_symbols, lib  # noqa: F401

__all__ = ["GinkgoError", "declared_symbols", "lib"]
