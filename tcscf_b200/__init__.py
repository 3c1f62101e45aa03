"""tcscf_b200: B200-native (sm_100a) grid-quadrature Fock build behind tcscf's integral / SCF interface."""
from . import basis, ffi, grids  # noqa: F401
from .api import (  # noqa: F401
    ConvergenceError,
    Context,
    LinearAlgebraError,
    QMCGrid,
    RCSHartreeFock,
    UOSHartreeFock,
    computeF,
    computeV,
    fock_build,
    fock_build_precomputed,
    overlap_core,
    overlap_core_quadrature,
)
