"""B200-native CUDA backend for the torchls block-sparse LM/GN inner loop.

Same modelling API as torchls (``Problem.add_residual``, ``Cost.factory`` /
``VarValues``, SO(3)/SE(3)/Sim(3) variables, Huber and custom losses, bounds,
``ConjugateGradientConfig``); every numerical step of ``solve`` runs in this
package's sm_100a kernels (``libtorchls_b200.so``, C ABI in
``include/torchls_b200.h``).
"""

from .batching import AutoBatchSize
from .cost import Cost
from .geometry import (
    SE2Var,
    SE3Var,
    Sim3Var,
    SO3Var,
    se3_exp,
    se3_log,
    se3_retract_jvp,
    sim3_exp,
    sim3_retract_jvp,
    so3_exp,
    so3_log,
    so3_retract_jvp,
)
from .linear_system import FixedLinearSystem, LADResult, LinearFactor, least_absolute_deviations
from .losses import HuberLoss, Loss
from .named import Problem
from .problem import AnalyzedLeastSquaresProblem, LeastSquaresProblem, Linearization
from .residuals import reprojection, se3_between, sim3_between
from .solvers import (
    BlockJacobiPreconditioner,
    ConjugateGradientConfig,
    NormalOperator,
    PCGResult,
    SolveSummary,
    TerminationConfig,
    TrustRegionConfig,
    block_jacobi,
    pcg,
)
from .sparse import BlockJacobian, CudaDiagonalPlan, CudaNormalPlan
from .variables import Var, VarValues

__all__ = [
    "AnalyzedLeastSquaresProblem",
    "AutoBatchSize",
    "BlockJacobiPreconditioner",
    "BlockJacobian",
    "ConjugateGradientConfig",
    "Cost",
    "FixedLinearSystem",
    "LADResult",
    "LinearFactor",
    "CudaDiagonalPlan",
    "CudaNormalPlan",
    "HuberLoss",
    "LeastSquaresProblem",
    "Linearization",
    "Loss",
    "NormalOperator",
    "PCGResult",
    "Problem",
    "SE2Var",
    "SE3Var",
    "SO3Var",
    "Sim3Var",
    "SolveSummary",
    "TerminationConfig",
    "TrustRegionConfig",
    "Var",
    "VarValues",
    "block_jacobi",
    "least_absolute_deviations",
    "pcg",
    "reprojection",
    "se3_between",
    "se3_exp",
    "se3_log",
    "se3_retract_jvp",
    "sim3_between",
    "sim3_exp",
    "sim3_retract_jvp",
    "so3_exp",
    "so3_log",
    "so3_retract_jvp",
]
__version__ = "0.1.0"
