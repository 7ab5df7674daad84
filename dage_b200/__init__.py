"""dage_b200: B200-native grid-based Coulomb/Helmholtz operator path of DAGE.

All arithmetic happens in ``libdagegpu.so`` (hand-written sm_100a CUDA
behind the C ABI declared in ``include/dage_gpu.h``); this package is the
host-side mirror of the reference's Operator3D/Function3D interface.
"""
from ._capi import DageError, load  # noqa: F401
from .operators import (  # noqa: F401
    Bubbles,
    Coulomb3D,
    GBFMMBatch,
    GBFMMCoulomb3D,
    GBFMMHelmholtz3D,
    GaussQuad,
    Grid1D,
    Grid3D,
    Helmholtz3D,
    Operator3D,
    apply_batched,
    cart2sph_table,
    cube_contaminants,
    dot,
    integrate,
    multiply,
    set_tune_cache,
)

__all__ = ["Bubbles", "Coulomb3D", "GBFMMBatch", "GBFMMCoulomb3D", "GBFMMHelmholtz3D", "GaussQuad", "Grid1D", "Grid3D", "Helmholtz3D", "Operator3D",
           "DageError", "apply_batched", "cart2sph_table", "cube_contaminants", "dot", "integrate", "load", "multiply", "set_tune_cache"]
