"""filtergs_b200: B200-native (sm_100a) FilterGS differentiable tile rasterizer and LoD-cut filtering.

Public surface:
  filtergs_b200.diff_gaussian_rasterization_wodilate  drop-in for the reference operator package
  filtergs_b200._C                                      mirror of the reference extension module
  filtergs_b200.filtergs_cuda                           FilterGS compute_radius_v2 / gather_attributes mirrors
"""
import sys

__version__ = "0.1.0"


def install_dropin():
    """Register this package's modules under the reference's import names
    (diff_gaussian_rasterization_wodilate, ._C) so unmodified callers import them."""
    from . import _C, diff_gaussian_rasterization_wodilate as dgr
    sys.modules.setdefault("diff_gaussian_rasterization_wodilate", dgr)
    sys.modules.setdefault("diff_gaussian_rasterization_wodilate._C", _C)
    return dgr
