"""tenet_b200: B200-native symmetric block-sparse tensor backend.

The hot path of TeNeT (fusion-tree recoupling transforms, per-coupled-sector
block contraction, blockwise factorisation) as hand-written sm_100a CUDA
kernels behind the C ABI of ``include/tenet_b200.h``.  The host structure
compiler (sectors, fusion trees, layouts, F/R/B recoupling coefficients) is
C++ in the same shared library; this package is the Python mirror of the
reference's typed facade over that ABI.
"""

from . import _lib, providers  # noqa: F401
from .typed import (  # noqa: F401
    FermionParityFusionRule,
    FusionRule,
    GradedSpace,
    HomSpace,
    Runtime,
    SU2FusionRule,
    TableFusionRule,
    TensorMap,
    Truncation,
    U1FusionRule,
    Z2FusionRule,
    product,
)

__version__ = "0.1.0"
