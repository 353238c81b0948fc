"""B200-native (sm_100a) explicit Gaussian and Beta CT operators.

Public surface of the reference's ``r2splat`` package (``r2splat/__init__.py:5-20``):
``rasterize_fwd``, ``rasterize_bwd``, ``voxelize_fwd``, ``voxelize_bwd`` and
``ParameterGradients``; the low-level operators live in ``r2splat_b200.cuda``.
"""

__version__ = "0.1.0"

from .explicit import (
    ParameterGradients,
    rasterize_bwd,
    rasterize_fwd,
    voxelize_bwd,
    voxelize_fwd,
)

__all__ = [
    "__version__",
    "rasterize_fwd",
    "rasterize_bwd",
    "voxelize_fwd",
    "voxelize_bwd",
    "ParameterGradients",
]
