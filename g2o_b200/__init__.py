"""B200-native backend for g2o's Gauss-Newton / Levenberg-Marquardt iteration
over a BlockSolver (bundle adjustment with Schur complement and block-Jacobi
PCG, pose graphs with Cholesky), behind the C-ABI of include/g2o_cuda.h.

The compute path is libg2o_b200.so (CUDA for sm_100a, built in-tree by
``python -m g2o_b200.build``). ``g2o_b200.backend`` is the host-side mirror
of g2o's SparseOptimizer / OptimizationAlgorithmFactory over that ABI.
"""
from . import abi  # noqa: F401

__all__ = ["abi", "backend", "synth", "build"]
