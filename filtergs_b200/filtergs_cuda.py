"""Mirrors of the FilterGS JIT modules (FilterGS/cuda/*.py and their kernels).

  compute_radius_module.compute_radius / .compute_visibility_radius
      FilterGS/cuda/compute_radius_kernel_v2.cu:355-435
  compute_visibility_radius(...)      FilterGS/cuda/compute_radius.py:23-45
  gather_attributes(...)              FilterGS/cuda/gather_attributes.py:20-42
  gather_attributes_cuda(...)         FilterGS/cuda/gather_attributes_kernel.cu:70-145

Same argument order, defaults and return types; the work runs in
libfiltergs_b200.so on torch's current stream.
"""
import ctypes as C

import torch

from ._lib import call


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None or t.numel() == 0 else C.c_void_p(t.data_ptr())


def _f32(t):
    return t.contiguous() if t.dtype == torch.float32 else t.float().contiguous()


class _ComputeRadiusModule:
    """The `compute_radius_v2` extension module object."""

    @staticmethod
    def compute_radius(means3D, scales, rotations, projmatrix, viewmatrix, focal_x, focal_y, tan_fovx, tan_fovy):
        P = int(means3D.shape[0])
        radii = torch.zeros(P, dtype=means3D.dtype, device=means3D.device)
        if P:
            call("fgs_compute_radius_v2", P, _p(_f32(means3D)), _p(_f32(scales)), _p(_f32(rotations)),
                 _p(_f32(projmatrix)), _p(_f32(viewmatrix)), float(focal_x), float(focal_y), float(tan_fovx),
                 float(tan_fovy), _p(radii), _s())
        return radii

    @staticmethod
    def compute_visibility_radius(means3D, scales, rotations, projmatrix, viewmatrix, tree_node_index,
                                  ancestor_path, focal_x, focal_y, tan_fovx, tan_fovy, padding, radius_max,
                                  radius_filter_threshold):
        P = int(means3D.shape[0])
        dev = means3D.device
        mask = torch.zeros(P, dtype=torch.bool, device=dev)
        radius2d = torch.full((P,), -1.0, dtype=torch.float32, device=dev)
        depth = torch.zeros(P, dtype=torch.float32, device=dev)
        L = int(ancestor_path.shape[1]) if ancestor_path.dim() == 2 else 0
        if P:
            call("fgs_visibility_radius", P, _p(_f32(means3D)), _p(_f32(scales)), _p(_f32(rotations)),
                 _p(_f32(projmatrix)), _p(_f32(viewmatrix)), _p(tree_node_index.to(torch.int32).contiguous()),
                 _p(ancestor_path.to(torch.int32).contiguous()), L, float(focal_x), float(focal_y), float(tan_fovx),
                 float(tan_fovy), float(padding), float(radius_max), float(radius_filter_threshold), _p(mask),
                 _p(radius2d), _p(depth), _s())
        return mask, radius2d, depth


compute_radius_module = _ComputeRadiusModule()


def compute_visibility_radius(means3d, scales, rotations, projmatrix, viewmatrix, tree_node_index, ancestor_path,
                              focal_x, focal_y, tan_fovx, tan_fovy, radius_max, padding=0.05,
                              radius_filter_threshold=100.0):
    """Visibility mask, 2D radius and NDC depth with the LoD tree rule (FilterGS/cuda/compute_radius.py:23-45)."""
    tensors = (means3d, scales, rotations, projmatrix, viewmatrix, tree_node_index, ancestor_path)
    if not all(t.is_cuda for t in tensors):
        raise ValueError("All input tensors must be CUDA tensors")
    return compute_radius_module.compute_visibility_radius(
        means3d, scales, rotations, projmatrix, viewmatrix, tree_node_index, ancestor_path, float(focal_x),
        float(focal_y), float(tan_fovx), float(tan_fovy), float(padding), float(radius_max),
        float(radius_filter_threshold))


def gather_attributes_cuda(index, xyz, scaling, rotation, opacity, colors, shs_opt=None):
    """gather_attributes_kernel.cu:70-145: list of gathered tensors (5, or 6 with shs)."""
    for name, t in (("index", index), ("xyz", xyz), ("scaling", scaling), ("rotation", rotation),
                    ("opacity", opacity), ("colors", colors)):
        if not t.is_cuda:
            raise RuntimeError(f"{name} must be CUDA tensor")
    idx = index.contiguous()
    N = int(idx.shape[0])
    xyz, scaling, rotation, opacity, colors = (t.contiguous() for t in (xyz, scaling, rotation, opacity, colors))
    o = [torch.empty(N, 3, dtype=xyz.dtype, device=xyz.device),
         torch.empty(N, 3, dtype=scaling.dtype, device=xyz.device),
         torch.empty(N, 4, dtype=rotation.dtype, device=xyz.device),
         torch.empty(N, 1, dtype=torch.float32, device=xyz.device),
         torch.empty(N, 3, dtype=colors.dtype, device=xyz.device)]
    shs = None
    coeffs = channels = 0
    if shs_opt is not None:
        if not shs_opt.is_cuda:
            raise RuntimeError("shs must be CUDA tensor")
        shs = shs_opt.contiguous()
        coeffs, channels = int(shs.shape[1]), int(shs.shape[2])
        o.append(torch.empty(N, coeffs, channels, dtype=shs.dtype, device=xyz.device))
    if N:
        call("fgs_gather_attributes", N, _p(idx), _p(xyz), _p(scaling), _p(rotation), _p(opacity), _p(colors),
             _p(shs), coeffs, channels, _p(o[0]), _p(o[1]), _p(o[2]), _p(o[3]), _p(o[4]),
             _p(o[5]) if shs is not None else None, _s())
    return o


def gather_attributes(index, xyz, scaling, rotation, opacity, colors, shs=None):
    """FilterGS/cuda/gather_attributes.py:20-42: dict of gathered rows."""
    for t in [index, xyz, scaling, rotation, opacity, colors] + ([shs] if shs is not None else []):
        assert t.is_cuda, "All input tensors must be CUDA tensors"
    if index.dtype != torch.long:
        index = index.to(dtype=torch.long)
    out = gather_attributes_cuda(index.contiguous(), xyz, scaling, rotation, opacity, colors, shs)
    keys = ["xyz", "scaling", "rotation", "opacity", "colors"]
    result = {k: out[i] for i, k in enumerate(keys)}
    if shs is not None:
        result["shs"] = out[-1]
    return result


__all__ = ["compute_radius_module", "compute_visibility_radius", "gather_attributes", "gather_attributes_cuda"]
