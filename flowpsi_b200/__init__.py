"""B200-native implicit residual-and-relaxation path of the flowPsi solver.

The compute path is the CUDA library ``libfpsi.so`` (sm_100a) behind the C ABI
of ``include/fpsi.h``; this package is its Python host side.
"""
from ._native import FpsiError, lib  # noqa: F401
from .solver import (  # noqa: F401
    FlowPsi,
    GeneratedMesh,
    bc,
    default_params,
    inviscid_riemann_flux,
    roe_jacobian,
)
from . import cases  # noqa: F401
