"""Python operator API of the rasterizer, a drop-in for the reference package
diff_gaussian_rasterization_wodilate (antialias/diff_gaussian_rasterization_wodilate/__init__.py).

GaussianRasterizationSettings, GaussianRasterizer, rasterize_gaussians and
_RasterizeGaussians keep the reference's field names, defaults, argument
checks, return arity and the `latest_stats` dictionary.  Two settings fields
are added at the end with defaults that keep the reference behaviour:

  filter3d_scale  3D (Mip-Splatting style) filter, cov3D += (s * z / focal)^2 I; 0 = off
  backward_mode   "ref_compat" (the reference backward, +0.3 dilation) or
                  "consistent" (the exact derivative of the forward as computed)
"""
from typing import NamedTuple

import torch
import torch.nn as nn

from . import _C


def cpu_deep_copy_tuple(input_tuple):
    copied = [item.cpu().clone() if isinstance(item, torch.Tensor) else item for item in input_tuple]
    return tuple(copied)


def rasterize_gaussians(means3D, means2D, sh, colors_precomp, opacities, scales, rotations, cov3Ds_precomp,
                        raster_settings, use_filter=True, ogfs_epsilon_scale=0.2, ogfs_epsilon_max=0.2,
                        ogfs_energy_floor=0.05, ogfs_radius_ratio_min=0.7, ogfs_enable_stats=True):
    """wodilate/__init__.py:21-54"""
    return _RasterizeGaussians.apply(means3D, means2D, sh, colors_precomp, opacities, scales, rotations,
                                     cov3Ds_precomp, raster_settings, use_filter, float(ogfs_epsilon_scale),
                                     float(ogfs_epsilon_max), float(ogfs_energy_floor), float(ogfs_radius_ratio_min),
                                     bool(ogfs_enable_stats))


class _RasterizeGaussians(torch.autograd.Function):
    """wodilate/__init__.py:56-191"""
    _last_stats = None

    @staticmethod
    def forward(ctx, means3D, means2D, sh, colors_precomp, opacities, scales, rotations, cov3Ds_precomp,
                raster_settings, use_filter, ogfs_epsilon_scale, ogfs_epsilon_max, ogfs_energy_floor,
                ogfs_radius_ratio_min, ogfs_enable_stats):
        filter3d = float(getattr(raster_settings, "filter3d_scale", 0.0))
        args = (raster_settings.bg, means3D, colors_precomp, opacities, scales, rotations,
                raster_settings.scale_modifier, cov3Ds_precomp, raster_settings.viewmatrix,
                raster_settings.projmatrix, raster_settings.tanfovx, raster_settings.tanfovy,
                raster_settings.image_height, raster_settings.image_width, sh, raster_settings.sh_degree,
                raster_settings.campos, raster_settings.prefiltered, use_filter, raster_settings.debug,
                ogfs_epsilon_scale, ogfs_epsilon_max, ogfs_energy_floor, ogfs_radius_ratio_min, ogfs_enable_stats)
        if raster_settings.debug:
            cpu_args = cpu_deep_copy_tuple(args)
            try:
                out = _C.rasterize_gaussians(*args, filter3d_scale=filter3d)
            except Exception as ex:
                torch.save(cpu_args, "snapshot_fw.dump")
                print("\nAn error occured in forward. Please forward snapshot_fw.dump for debugging.")
                raise ex
        else:
            out = _C.rasterize_gaussians(*args, filter3d_scale=filter3d)
        num_rendered, color, point_id, point_weight_pixel, point_weight, radii, geomBuffer, binningBuffer, \
            imgBuffer, stats = out
        _RasterizeGaussians._last_stats = stats
        ctx.raster_settings = raster_settings
        ctx.num_rendered = num_rendered
        ctx.use_filter = bool(use_filter)
        ctx.save_for_backward(colors_precomp, means3D, scales, rotations, cov3Ds_precomp, radii, sh, geomBuffer,
                              binningBuffer, imgBuffer)
        return color, radii, point_id, point_weight_pixel, point_weight

    @staticmethod
    def backward(ctx, grad_out_color, radii, point_id, point_weight_pixel, point_weight):
        num_rendered = ctx.num_rendered
        rs = ctx.raster_settings
        colors_precomp, means3D, scales, rotations, cov3Ds_precomp, radii, sh, geomBuffer, binningBuffer, \
            imgBuffer = ctx.saved_tensors
        args = (rs.bg, means3D, radii, colors_precomp, scales, rotations, rs.scale_modifier, cov3Ds_precomp,
                rs.viewmatrix, rs.projmatrix, rs.tanfovx, rs.tanfovy, grad_out_color, sh, rs.sh_degree, rs.campos,
                geomBuffer, num_rendered, binningBuffer, imgBuffer, rs.debug)
        kw = dict(use_filter=ctx.use_filter, backward_mode=getattr(rs, "backward_mode", "ref_compat"),
                  filter3d_scale=float(getattr(rs, "filter3d_scale", 0.0)))
        if rs.debug:
            cpu_args = cpu_deep_copy_tuple(args)
            try:
                grads = _C.rasterize_gaussians_backward(*args, **kw)
            except Exception as ex:
                torch.save(cpu_args, "snapshot_bw.dump")
                print("\nAn error occured in backward. Writing snapshot_bw.dump for debugging.\n")
                raise ex
        else:
            grads = _C.rasterize_gaussians_backward(*args, **kw)
        grad_means2D, grad_colors_precomp, grad_opacities, grad_means3D, grad_cov3Ds_precomp, grad_sh, \
            grad_scales, grad_rotations = grads
        if grad_colors_precomp.shape[-1] > 3:
            grad_colors_precomp = grad_colors_precomp[:, :3]
        return (grad_means3D, grad_means2D, grad_sh, grad_colors_precomp, grad_opacities, grad_scales,
                grad_rotations, grad_cov3Ds_precomp, None, None, None, None, None, None, None)


class GaussianRasterizationSettings(NamedTuple):
    """wodilate/__init__.py:193-210 (+ filter3d_scale, backward_mode)."""
    image_height: int
    image_width: int
    tanfovx: float
    tanfovy: float
    bg: torch.Tensor
    scale_modifier: float
    viewmatrix: torch.Tensor
    projmatrix: torch.Tensor
    sh_degree: int
    campos: torch.Tensor
    prefiltered: bool
    debug: bool
    ogfs_epsilon_scale: float = 0.2
    ogfs_epsilon_max: float = 0.2
    ogfs_energy_floor: float = 0.05
    ogfs_radius_ratio_min: float = 0.7
    ogfs_enable_stats: bool = True
    filter3d_scale: float = 0.0
    backward_mode: str = "ref_compat"


def parse_stats(stats_tensor):
    """The `latest_stats` dictionary of wodilate/__init__.py:306-344."""
    if stats_tensor is None or not torch.is_tensor(stats_tensor):
        return None
    s = stats_tensor.detach().cpu().tolist()
    if len(s) < 16:
        return None
    d = {'bar_g': float(s[0]), 'avg_kv_per_gaussian': float(s[1]), 'avg_kv_per_tile': float(s[2]),
         'num_kv_pairs': float(s[3]), 'num_tiles': float(s[4]), 'num_gaussians': float(s[5])}
    d['used_kv_pairs'] = float(s[6])
    d['unused_kv_pairs'] = float(s[7])
    num_kpc_bins = int(s[8])
    d['num_kpc_bins'] = num_kpc_bins
    rem = s[9:]
    num_tiles = int(d['num_tiles'])
    kpc_slots = 0
    if len(rem) >= 2 * num_tiles:
        kpc_slots = (len(rem) - 2 * num_tiles) // 2
    if kpc_slots > 0:
        part = rem[:2 * kpc_slots]
        d['kpc_edges'] = part[:kpc_slots][:num_kpc_bins]
        d['kpc_hist'] = part[kpc_slots:][:num_kpc_bins]
        rem = rem[2 * kpc_slots:]
    if rem and num_tiles > 0:
        if len(rem) >= num_tiles:
            d['tile_ratio'] = rem[:num_tiles]
            rem = rem[num_tiles:]
        if len(rem) >= num_tiles:
            d['tile_total_kv'] = rem[:num_tiles]
    return d


class GaussianRasterizer(nn.Module):
    """wodilate/__init__.py:212-345"""

    def __init__(self, raster_settings):
        super().__init__()
        self.raster_settings = raster_settings
        self.latest_stats = None

    def compute_radius(self, positions, scales, rotations):
        with torch.no_grad():
            rs = self.raster_settings
            return _C.compute_radius(positions, scales, rotations, rs.viewmatrix, rs.projmatrix, rs.tanfovx,
                                     rs.tanfovy, rs.image_height, rs.image_width)

    def markVisible(self, positions):
        with torch.no_grad():
            rs = self.raster_settings
            return _C.mark_visible(positions, rs.viewmatrix, rs.projmatrix)

    def forward(self, means3D, means2D, opacities, shs=None, colors_precomp=None, scales=None, rotations=None,
                cov3D_precomp=None, use_filter=True, ogfs_epsilon_scale=None, ogfs_epsilon_max=None,
                ogfs_energy_floor=None, ogfs_radius_ratio_min=None, ogfs_enable_stats=None):
        rs = self.raster_settings
        eps_scale = rs.ogfs_epsilon_scale if ogfs_epsilon_scale is None else ogfs_epsilon_scale
        eps_max = rs.ogfs_epsilon_max if ogfs_epsilon_max is None else ogfs_epsilon_max
        energy_floor = rs.ogfs_energy_floor if ogfs_energy_floor is None else ogfs_energy_floor
        radius_min = rs.ogfs_radius_ratio_min if ogfs_radius_ratio_min is None else ogfs_radius_ratio_min
        enable_stats = rs.ogfs_enable_stats if ogfs_enable_stats is None else ogfs_enable_stats

        if (shs is None and colors_precomp is None) or (shs is not None and colors_precomp is not None):
            raise Exception('Please provide excatly one of either SHs or precomputed colors!')
        if ((scales is None or rotations is None) and cov3D_precomp is None) or \
                ((scales is not None or rotations is not None) and cov3D_precomp is not None):
            raise Exception('Please provide exactly one of either scale/rotation pair or precomputed 3D covariance!')
        if shs is None:
            shs = torch.Tensor([])
        if colors_precomp is None:
            colors_precomp = torch.Tensor([])
        if scales is None:
            scales = torch.Tensor([])
        if rotations is None:
            rotations = torch.Tensor([])
        if cov3D_precomp is None:
            cov3D_precomp = torch.Tensor([])

        result = rasterize_gaussians(means3D, means2D, shs, colors_precomp, opacities, scales, rotations,
                                     cov3D_precomp, rs, use_filter, float(eps_scale), float(eps_max),
                                     float(energy_floor), float(radius_min), bool(enable_stats))
        self.latest_stats = parse_stats(getattr(_RasterizeGaussians, "_last_stats", None))
        return result
