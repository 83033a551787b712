"""Drop-in module with the reference package's name and contents
(antialias/diff_gaussian_rasterization_wodilate/__init__.py).

    from filtergs_b200 import diff_gaussian_rasterization_wodilate as dgr

or install it under its reference name with filtergs_b200.install_dropin().
"""
from .. import _C  # noqa: F401
from ..rasterization import (GaussianRasterizationSettings, GaussianRasterizer, _RasterizeGaussians,  # noqa: F401
                             cpu_deep_copy_tuple, rasterize_gaussians)

__all__ = ["GaussianRasterizationSettings", "GaussianRasterizer", "rasterize_gaussians", "_RasterizeGaussians",
           "_C", "cpu_deep_copy_tuple"]
