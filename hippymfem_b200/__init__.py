"""hippymfem_b200: B200-native kernels for hIPPyMFEM's Q2 log-conductivity assembly and
Hessian-action path, behind the reference's problem/form API.

The compute path is ``libhippymfem_b200.so`` (hand-written sm_100a CUDA behind the C ABI
of ``include/hippymfem_b200.h``); importing this package fails if it is not built.
"""

from ._lib import HM_FP32, HM_FP64, NotConvergedError  # noqa: F401  (loads the library)
from .mesh import BoxMesh, DirichletBC, Q2Space  # noqa: F401
from .modeling import (BiLaplacianPrior, DeviceCSR, DiscreteStateObservation,  # noqa: F401
                       Model, PointwiseStateObservation, ReducedHessian,
                       device_observation_operator, observation_operator)
from .pattern import LatticePattern, build_tables  # noqa: F401
from .problem import ADJOINT, NVAR, PARAMETER, STATE, PDEVariationalProblem  # noqa: F401
from .sparse import CSRBlock, MatrixFreeJacobian, MixedPCGSolver, PCGSolver  # noqa: F401

__version__ = "0.1.0"
