"""B200-native vertex-patch Schwarz multigrid for continuous Q_k (2D/3D).

The compute path is libtps.so (C++ host + sm_100a CUDA kernels) behind the C
ABI of include/tps.h; this package mirrors the reference's operator API over
that ABI.
"""
from .api import (BatchSolver, LaplaceOperator, MGTransferCUDA, MultigridSolvers, PatchSmoother,
                  PoissonProblem, SolveReport, split_cells)
from ._lib import TpsError
from .autograd import PoissonSolve

__all__ = ["BatchSolver", "LaplaceOperator", "MGTransferCUDA", "MultigridSolvers", "PatchSmoother",
           "PoissonProblem", "PoissonSolve", "SolveReport", "TpsError", "split_cells"]
