"""B200-native (sm_100a) hot path of the higher-order embedded FEM method.

Per-element hyperelastic force / tangent stiffness (Stable Neo-Hookean, StVK;
Tet10 and embedded Hex27), atomic-free colored CSR scatter assembly, and the
Schwarz-preconditioned CG solve inside the backward-Euler Newton loop, all as
CUDA kernels behind the C ABI of include/hoefem.h (libhoefem.so).  This
package is the Python host mirror of the reference's fenris / hamilton2 /
simulation_toolbox interfaces for that path.
"""
from ._capi import HoefemError, ELEM_HEX27, ELEM_TET10, LIB_PATH  # noqa: F401
from .materials import LameParameters, StableNeoHookeanMaterial, StVKMaterial, YoungPoisson  # noqa: F401
from .model import EmbeddedModel3d, NodalModel3d  # noqa: F401
from .solver import (  # noqa: F401
    BatchedNewtonCgIntegrator3d,
    CgOutput,
    ConjugateGradient,
    DiagonalPreconditioner,
    NewtonCgIntegrator3d,
    RelativeResidualCriterion,
    SchwarzPreconditioner,
    SchwarzPreconditionerComponent,
    SolveError,
    SolveErrorKind,
)
from .learned import LearnedCoarseCorrection  # noqa: F401
from .embedding import (  # noqa: F401
    EmbedOptions,
    EmbeddedQuadrature,
    StabilizationOptions,
    embed_mesh_3d,
    embed_quadrature_3d,
    simplify_quadrature,
    tet_quadrature_strength,
)
from . import scenes  # noqa: F401
