"""Host-side mirror of the reference extension module `_C`
(antialias/ext.cpp:17-49, antialias/rasterize_points.cu:36-318).

Same function names, argument order, keyword defaults and return tuples as
diff_gaussian_rasterization_wodilate._C.  Tensors are handed to the C ABI of
libfiltergs_b200.so as raw device pointers on torch's current stream; torch
only allocates the outputs and the three opaque workspace buffers.

Extensions beyond the reference (keyword-only, defaults keep reference
behaviour): `filter3d_scale` on rasterize_gaussians; `use_filter`,
`backward_mode` and `filter3d_scale` on rasterize_gaussians_backward.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import RasterArgs, call, lib

NUM_CHANNELS = 3
KPC_SLOTS = _lib.FGS_STATS_SLOTS
BACKWARD_MODES = {"ref_compat": _lib.FGS_BACKWARD_REF_COMPAT, "consistent": _lib.FGS_BACKWARD_CONSISTENT}


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    """Device pointer of a float/int tensor, or None for an absent (empty) input."""
    if t is None or t.numel() == 0:
        return None
    return C.c_void_p(t.data_ptr())


def _dev_f32(t, device, name):
    """An input as contiguous float32 on `device` (empty tensors stay empty = absent)."""
    if t is None or t.numel() == 0:
        return None
    if t.dtype != torch.float32:
        raise RuntimeError(f"{name} must be a float32 tensor (got {t.dtype})")
    if t.device != device:
        t = t.to(device)
    return t.contiguous()


def _args(P, D, M, W, H, bg, means3D, sh, colors, opacity, scales, scale_modifier, rotations, cov3D, view, proj,
          campos, tanx, tany, prefiltered, use_filter, eps_scale, eps_max, energy_floor, ratio_min, stats,
          filter3d_scale):
    a = RasterArgs()
    a.P, a.D, a.M, a.width, a.height = int(P), int(D), int(M), int(W), int(H)
    a.background, a.means3D, a.shs, a.colors_precomp = _ptr(bg), _ptr(means3D), _ptr(sh), _ptr(colors)
    a.opacities, a.scales, a.rotations, a.cov3D_precomp = _ptr(opacity), _ptr(scales), _ptr(rotations), _ptr(cov3D)
    a.scale_modifier = float(scale_modifier)
    a.viewmatrix, a.projmatrix, a.campos = _ptr(view), _ptr(proj), _ptr(campos)
    a.tan_fovx, a.tan_fovy = float(tanx), float(tany)
    a.prefiltered, a.use_filter = int(bool(prefiltered)), int(bool(use_filter))
    a.ogfs_epsilon_scale, a.ogfs_epsilon_max = float(eps_scale), float(eps_max)
    a.ogfs_energy_floor, a.ogfs_radius_ratio_min = float(energy_floor), float(ratio_min)
    a.ogfs_enable_stats = int(bool(stats))
    a.filter3d_scale = float(filter3d_scale)
    return a


def _num_tiles(W, H):
    return ((W + 15) // 16) * ((H + 15) // 16)


def rasterize_gaussians(background, means3D, colors, opacity, scales, rotations, scale_modifier, cov3D_precomp,
                        viewmatrix, projmatrix, tan_fovx, tan_fovy, image_height, image_width, sh, degree, campos,
                        prefiltered, use_filter, debug=False, ogfs_epsilon_scale=0.2, ogfs_epsilon_max=0.2,
                        ogfs_energy_floor=0.05, ogfs_radius_ratio_min=0.7, ogfs_enable_stats=True, *,
                        filter3d_scale=0.0):
    """RasterizeGaussiansCUDA (rasterize_points.cu:36-179).

    Returns (num_rendered, out_color[3,H,W], point_id[H,W] i32, point_weight_pixel[H,W],
    point_weight[P], radii[P] i32, geomBuffer u8, binningBuffer u8, imgBuffer u8, stats f64 cpu)."""
    if means3D.ndim != 2 or means3D.shape[1] != 3:
        raise RuntimeError("means3D must have dimensions (num_points, 3)")
    dev = means3D.device
    if dev.type != "cuda":
        raise RuntimeError("means3D must be a CUDA tensor")
    P, H, W = int(means3D.shape[0]), int(image_height), int(image_width)
    fo = dict(device=dev, dtype=torch.float32)
    io = dict(device=dev, dtype=torch.int32)
    u8 = dict(device=dev, dtype=torch.uint8)
    T = _num_tiles(W, H)
    if P == 0:
        stats = torch.zeros(9 + 2 * KPC_SLOTS, dtype=torch.float64)
        return (0, torch.zeros(NUM_CHANNELS, H, W, **fo), torch.zeros(H, W, **io), torch.zeros(H, W, **fo),
                torch.zeros(0, **fo), torch.zeros(0, **io), torch.empty(0, **u8), torch.empty(0, **u8),
                torch.empty(0, **u8), stats)
    means3D = _dev_f32(means3D, dev, "means3D")
    opacity = _dev_f32(opacity, dev, "opacity")
    colors = _dev_f32(colors, dev, "colors")
    scales = _dev_f32(scales, dev, "scales")
    rotations = _dev_f32(rotations, dev, "rotations")
    cov3D_precomp = _dev_f32(cov3D_precomp, dev, "cov3D_precomp")
    sh = _dev_f32(sh, dev, "sh")
    bg = _dev_f32(background, dev, "background")
    view = _dev_f32(viewmatrix, dev, "viewmatrix")
    proj = _dev_f32(projmatrix, dev, "projmatrix")
    cam = _dev_f32(campos, dev, "campos")
    M = int(sh.shape[1]) if sh is not None else 0
    a = _args(P, degree, M, W, H, bg, means3D, sh, colors, opacity, scales, scale_modifier, rotations,
              cov3D_precomp, view, proj, cam, tan_fovx, tan_fovy, prefiltered, use_filter, ogfs_epsilon_scale,
              ogfs_epsilon_max, ogfs_energy_floor, ogfs_radius_ratio_min, ogfs_enable_stats, filter3d_scale)
    L = lib()
    geom = torch.empty(int(L.fgs_geom_bytes(P)), **u8)
    img = torch.empty(int(L.fgs_image_bytes(W, H)), **u8)
    radii = torch.empty(P, **io)
    stream = _stream()
    K = C.c_longlong(0)
    call("fgs_forward_preprocess", C.byref(a), _ptr(geom), _ptr(img), _ptr(radii), C.byref(K), stream)
    K = int(K.value)
    binning = torch.empty(int(L.fgs_binning_bytes(K, P)), **u8)
    out_color = torch.empty(NUM_CHANNELS, H, W, **fo)
    point_id = torch.empty(H, W, **io)
    pw_pixel = torch.empty(H, W, **fo)
    point_weight = torch.empty(P, **fo)
    n_stats = 9 + 2 * KPC_SLOTS + (2 * T if (ogfs_enable_stats and K > 0) else 0)
    stats = np.zeros(n_stats, np.float64)
    call("fgs_forward_render", C.byref(a), _ptr(geom), _ptr(img), _ptr(binning), C.c_longlong(K), _ptr(radii),
         _ptr(out_color), _ptr(point_id), _ptr(pw_pixel), _ptr(point_weight),
         stats.ctypes.data_as(C.c_void_p), n_stats, stream)
    if debug:
        call("fgs_check", _ptr(geom), stream)
    return (K, out_color, point_id, pw_pixel, point_weight, radii, geom, binning, img, torch.from_numpy(stats))


def rasterize_gaussians_backward(background, means3D, radii, colors, scales, rotations, scale_modifier,
                                 cov3D_precomp, viewmatrix, projmatrix, tan_fovx, tan_fovy, dL_dout_color, sh,
                                 degree, campos, geomBuffer, R, binningBuffer, imageBuffer, debug=False, *,
                                 use_filter=True, backward_mode="ref_compat", filter3d_scale=0.0):
    """RasterizeGaussiansBackwardCUDA (rasterize_points.cu:181-260).

    Returns (dL_dmeans2D[P,3], dL_dcolors[P,3], dL_dopacity[P,1], dL_dmeans3D[P,3], dL_dcov3D[P,6],
    dL_dsh[P,M,3], dL_dscales[P,3], dL_drotations[P,4])."""
    dev = means3D.device
    P = int(means3D.shape[0])
    H, W = int(dL_dout_color.shape[1]), int(dL_dout_color.shape[2])
    sh = _dev_f32(sh, dev, "sh")
    M = int(sh.shape[1]) if sh is not None else 0
    fo = dict(device=dev, dtype=torch.float32)
    g_m2 = torch.empty(P, 3, **fo)
    g_col = torch.empty(P, NUM_CHANNELS, **fo)
    g_op = torch.empty(P, 1, **fo)
    g_m3 = torch.empty(P, 3, **fo)
    g_cov = torch.empty(P, 6, **fo)
    g_sh = torch.empty(P, M, 3, **fo)
    g_sc = torch.empty(P, 3, **fo)
    g_rot = torch.empty(P, 4, **fo)
    if P == 0:
        return g_m2, g_col, g_op, g_m3, g_cov, g_sh, g_sc, g_rot
    if backward_mode not in BACKWARD_MODES:
        raise ValueError(f"backward_mode must be one of {sorted(BACKWARD_MODES)}")
    g_conic = torch.empty(P, 4, **fo)
    means3D = _dev_f32(means3D, dev, "means3D")
    colors = _dev_f32(colors, dev, "colors")
    scales = _dev_f32(scales, dev, "scales")
    rotations = _dev_f32(rotations, dev, "rotations")
    cov3D_precomp = _dev_f32(cov3D_precomp, dev, "cov3D_precomp")
    dpix = _dev_f32(dL_dout_color, dev, "dL_dout_color")
    bg = _dev_f32(background, dev, "background")
    view = _dev_f32(viewmatrix, dev, "viewmatrix")
    proj = _dev_f32(projmatrix, dev, "projmatrix")
    cam = _dev_f32(campos, dev, "campos")
    radii = radii.contiguous() if radii is not None and radii.numel() else None
    a = _args(P, degree, M, W, H, bg, means3D, sh, colors, None, scales, scale_modifier, rotations, cov3D_precomp,
              view, proj, cam, tan_fovx, tan_fovy, False, use_filter, 0.2, 0.2, 0.05, 0.7, False, filter3d_scale)
    stream = _stream()
    call("fgs_backward", C.byref(a), _ptr(geomBuffer), _ptr(imageBuffer), _ptr(binningBuffer), C.c_longlong(int(R)),
         _ptr(radii), _ptr(dpix), _ptr(g_m2), _ptr(g_conic), _ptr(g_op), _ptr(g_col), _ptr(g_m3), _ptr(g_cov),
         _ptr(g_sh), _ptr(g_sc), _ptr(g_rot), BACKWARD_MODES[backward_mode], stream)
    if debug:
        call("fgs_check", _ptr(geomBuffer), stream)
    return g_m2, g_col, g_op, g_m3, g_cov, g_sh, g_sc, g_rot


def mark_visible(means3D, viewmatrix, projmatrix):
    """markVisible (rasterize_points.cu:299-318): bool[P], view-space z > 0.2."""
    dev = means3D.device
    P = int(means3D.shape[0])
    present = torch.zeros(P, dtype=torch.bool, device=dev)
    if P:
        call("fgs_mark_visible", P, _ptr(_dev_f32(means3D, dev, "means3D")), _ptr(_dev_f32(viewmatrix, dev, "view")),
             _ptr(_dev_f32(projmatrix, dev, "proj")), _ptr(present), _stream())
    return present


def compute_radius(means3D, scales, rotations, viewmatrix, projmatrix, tan_fovx, tan_fovy, image_height,
                   image_width):
    """compute_radius (rasterize_points.cu:263-296): 3-sigma screen radius, float32[P] (0 = culled)."""
    dev = means3D.device
    P = int(means3D.shape[0])
    radii = torch.zeros(P, dtype=torch.float32, device=dev)
    if P:
        call("fgs_compute_radius", P, int(image_height), int(image_width), _ptr(_dev_f32(means3D, dev, "means3D")),
             _ptr(_dev_f32(scales, dev, "scales")), _ptr(_dev_f32(rotations, dev, "rotations")),
             _ptr(_dev_f32(viewmatrix, dev, "view")), _ptr(_dev_f32(projmatrix, dev, "proj")), float(tan_fovx),
             float(tan_fovy), _ptr(radii), _stream())
    return radii


# ---------------------------------------------------------------- test accessors
def sorted_pairs(geomBuffer, binningBuffer, P, num_rendered):
    """Sorted 64-bit (tile|depth) keys (as int64 bit patterns) and Gaussian ids of a forward."""
    dev = geomBuffer.device
    keys = torch.empty(num_rendered, dtype=torch.int64, device=dev)
    vals = torch.empty(num_rendered, dtype=torch.int32, device=dev)
    if num_rendered:
        call("fgs_sorted_pairs", _ptr(geomBuffer), _ptr(binningBuffer), int(P), C.c_longlong(num_rendered),
             _ptr(keys), _ptr(vals), _stream())
    return keys, vals


def preprocess_outputs(geomBuffer, P):
    dev = geomBuffer.device
    fo = dict(device=dev, dtype=torch.float32)
    out = dict(means2D=torch.empty(P, 2, **fo), depths=torch.empty(P, **fo), conic_opacity=torch.empty(P, 4, **fo),
               rgb=torch.empty(P, 3, **fo), tiles_touched=torch.empty(P, dtype=torch.int32, device=dev))
    if P:
        call("fgs_preprocess_outputs", _ptr(geomBuffer), int(P), _ptr(out["means2D"]), _ptr(out["depths"]),
             _ptr(out["conic_opacity"]), _ptr(out["rgb"]), _ptr(out["tiles_touched"]), _stream())
    return out


def image_outputs(imgBuffer, W, H):
    dev = imgBuffer.device
    out = dict(final_T=torch.empty(H * W, dtype=torch.float32, device=dev),
               n_contrib=torch.empty(H * W, dtype=torch.int32, device=dev),
               ranges=torch.empty(_num_tiles(W, H), 2, dtype=torch.int32, device=dev))
    call("fgs_image_outputs", _ptr(imgBuffer), int(W), int(H), _ptr(out["final_T"]), _ptr(out["n_contrib"]),
         _ptr(out["ranges"]), _stream())
    return out
