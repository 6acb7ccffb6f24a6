"""B200-native hot path of one adaptive cycle of the space-time parabolic FEM of
Rsmeets99/DoubleAdapParabolicFEM: main-system assembly, block-preconditioned MINRES
and the equilibrated-flux estimator, as sm_100a CUDA kernels behind a C ABI
(include/apf_b200.h) with a Python mirror of the reference's call signatures."""
from .mesh import Restriction, SpaceTimeProblem, uniform_problem  # noqa: F401

__all__ = ["Restriction", "SpaceTimeProblem", "uniform_problem"]
