"""Per-view LoD selection on the device, in front of the rasterizer.

Two selection rules over a Gaussian tree (node arrays in the layout of
LoG/model/tensor_tree.py and apps/ancestor.py):

  FilterGS rule   compute_visibility_radius (FilterGS/cuda/compute_radius_kernel_v2.cu:231-353):
                  visible internal nodes with radius <= radius_max, visible leaves with no
                  visible internal ancestor of radius in (0, radius_max], minus radii above the
                  large-radius threshold.  FilterGS.prepare/get_all (FilterGS/filtergs.py:20-134).
  LoG cut rule    TensorTree.traverse (LoG/model/tensor_tree.py:133-187) with min_resolution_pixel,
                  then redundancy culling: drop radius < 1 px or sigmoid(opacity) < 1/255.

Both stay on the device: the mask is compacted with an ordered device scan,
the rows are gathered and activated in one kernel (exp scale, sigmoid
opacity, normalised quaternion, SH colour), and the traversal is a
level-synchronous frontier.  The only host synchronisation is reading the
selected count before the rasterizer is called.
"""
import ctypes as C

import torch

from . import _C
from ._lib import call, lib
from .filtergs_cuda import compute_visibility_radius


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None or t.numel() == 0 else C.c_void_p(t.data_ptr())


class TreeScene:
    """Raw (pre-activation) parameters of a Gaussian LoD tree on one device."""

    def __init__(self, xyz, log_scales, rotations, opacity_raw, features_dc, shs_rest, node_index, ancestor_path,
                 tree, roots, sh_degree=1, device="cuda"):
        t = lambda a, dt=torch.float32: torch.as_tensor(a).to(device=device, dtype=dt).contiguous()  # noqa: E731
        self.xyz, self.log_scales, self.rotations = t(xyz), t(log_scales), t(rotations)
        self.opacity_raw, self.features_dc = t(opacity_raw).reshape(-1), t(features_dc)
        self.shs_rest = t(shs_rest) if shs_rest is not None else None
        self.node_index = t(node_index, torch.int32)
        self.ancestor_path = t(ancestor_path, torch.int32)
        self.tree = t(tree, torch.int32)
        self.roots = t(roots, torch.int32)
        self.sh_degree = int(sh_degree)
        self.P = int(self.xyz.shape[0])
        self.cut_levels = _frontier_levels(self.roots, self.node_index, self.tree)

    @classmethod
    def from_arrays(cls, d, device="cuda"):
        return cls(d["xyz"], d["log_scales"], d["rotations"], d["opacity_raw"], d["features_dc"], d.get("shs_rest"),
                   d["node_index"], d["ancestor_path"], d["tree"], d["roots"], sh_degree=1, device=device)


def _frontier_levels(roots, node_index, tree, cap=30):
    """Non-empty frontiers of a level-by-level walk from the roots through every child (at most
    cap): a LoG cut never needs more levels, whatever the radii, since its frontiers are subsets
    of these and a level with an empty frontier changes nothing."""
    P = int(node_index.numel())
    rows = int(tree.shape[0]) if tree.dim() >= 1 else 0
    f = roots.long()
    levels = 0
    while levels < cap:
        f = f[(f >= 0) & (f < P)]
        if f.numel() == 0:
            break
        levels += 1
        ni = node_index[f].long()
        ni = ni[(ni >= 0) & (ni < rows)]
        ch = tree[ni].reshape(-1).long()
        f = ch[ch >= 0]
    return levels


def _focal(cam):
    return cam.W / (2.0 * cam.tanfovx), cam.H / (2.0 * cam.tanfovy)


def compact(mask):
    """Ordered int64 indices of a bool/uint8 mask; count stays on the device (int64 tensor [1])."""
    n = int(mask.numel())
    dev = mask.device
    idx = torch.empty(n, dtype=torch.int64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    scratch = torch.empty(int(lib().fgs_compact_scratch_bytes(n)) // 4 + 1, dtype=torch.int32, device=dev)
    call("fgs_compact_mask", n, _p(mask.contiguous().view(torch.uint8)), _p(idx), _p(cnt), _p(scratch), _s())
    return idx, cnt


def select_filtergs(scene, view, proj, cam, radius_max=1.5, padding=0.1, radius_filter_threshold=700.0):
    """FilterGS rule -> (index int64 buffer [P], count int64 [1] on device, mask, radius2d, depth)."""
    fx, fy = _focal(cam)
    mask, radius2d, depth = compute_visibility_radius(scene.xyz, scene.log_scales, scene.rotations, proj, view,
                                                      scene.node_index, scene.ancestor_path, fx, fy, cam.tanfovx,
                                                      cam.tanfovy, radius_max, padding, radius_filter_threshold)
    idx, cnt = compact(mask)
    return idx, cnt, mask, radius2d, depth


def node_radius(scene, view, proj, cam):
    """LoG node radius (v2 3-sigma kernel) from raw parameters."""
    fx, fy = _focal(cam)
    r = torch.empty(scene.P, dtype=torch.float32, device=scene.xyz.device)
    call("fgs_radius_raw", scene.P, _p(scene.xyz), _p(scene.log_scales), _p(scene.rotations), _p(view), _p(proj),
         float(fx), float(fy), float(cam.tanfovx), float(cam.tanfovy), _p(r), _s())
    return r


def log_cut(scene, radius, min_resolution_pixel=1.5, levels=30):
    """TensorTree.traverse order on the device -> (ids int32 buffer [P], count int32 [1] on device).
    levels caps the walk as traverse's 30 does; the tree's own depth caps it further (the levels
    past it find an empty frontier)."""
    levels = min(int(levels), getattr(scene, "cut_levels", int(levels)))
    dev = scene.xyz.device
    P = scene.P
    mc = int(scene.tree.shape[1]) if scene.tree.dim() == 2 else 1
    out = torch.empty(P, dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    nroots = int(scene.roots.numel())
    sb = int(lib().fgs_log_cut_scratch_bytes(P, nroots, mc, levels))
    scratch = torch.empty(sb // 4 + 1, dtype=torch.int32, device=dev)
    call("fgs_log_cut", P, _p(scene.roots), nroots, _p(scene.node_index), _p(scene.tree), mc, _p(radius),
         float(min_resolution_pixel), int(levels), _p(out), _p(cnt), _p(scratch), _s())
    return out, cnt


def cull(ids, count, radius, opacity_raw, min_px=1.0):
    """Keep ids with radius >= min_px and sigmoid(opacity) >= 1/255 -> (int64 [cap], count int64 [1])."""
    dev = ids.device
    cap = int(ids.numel())
    out = torch.empty(cap, dtype=torch.int64, device=dev)
    oc = torch.zeros(1, dtype=torch.int64, device=dev)
    scratch = torch.empty(int(lib().fgs_compact_scratch_bytes(cap)) // 4 + 1, dtype=torch.int32, device=dev)
    call("fgs_cull", _p(ids), _p(count), cap, _p(radius), _p(opacity_raw), float(min_px), _p(out), _p(oc),
         _p(scratch), _s())
    return out, oc


def select_logcut(scene, view, proj, cam, min_resolution_pixel=1.5, min_px=1.0, levels=30):
    """LoG cut + redundancy culling -> (index int64 buffer [P], count int64 [1] on device)."""
    r = node_radius(scene, view, proj, cam)
    ids, c = log_cut(scene, r, min_resolution_pixel, levels)
    return cull(ids, c, r, scene.opacity_raw, min_px)


def gather_activate(scene, index, count, campos, cap=None):
    """Gathered, activated rows (xyz, scaling, rotation, opacity, colors) of index[0..count)."""
    dev = scene.xyz.device
    N = int(index.numel()) if cap is None else int(cap)
    o = dict(xyz=torch.empty(N, 3, device=dev), scaling=torch.empty(N, 3, device=dev),
             rotation=torch.empty(N, 4, device=dev), opacity=torch.empty(N, 1, device=dev),
             colors=torch.empty(N, 3, device=dev))
    rest = scene.shs_rest
    rc = int(rest.shape[1]) if rest is not None else 0
    if N:
        call("fgs_gather_activate", N, _p(index), _p(count), _p(scene.xyz), _p(scene.log_scales), _p(scene.rotations),
             _p(scene.opacity_raw), _p(scene.features_dc), _p(rest), scene.sh_degree if rest is not None else 0, rc,
             _p(campos), _p(o["xyz"]), _p(o["scaling"]), _p(o["rotation"]), _p(o["opacity"]), _p(o["colors"]), _s())
    return o


def drop_invalid_rows(rows):
    """FilterGS.render's guard (FilterGS/filtergs.py:159-172): keep the rows whose attributes are all
    finite with min(scale) > 0 and opacity > 0, in order.  Rows are returned unchanged when none is
    dropped (the common case: one device flag read)."""
    dev = rows["xyz"].device
    n = int(rows["xyz"].shape[0])
    keep = torch.empty(n, dtype=torch.uint8, device=dev)
    dropped = torch.zeros(1, dtype=torch.int64, device=dev)
    call("fgs_rows_valid", n, _p(rows["xyz"]), _p(rows["scaling"]), _p(rows["rotation"]), _p(rows["opacity"]),
         _p(rows["colors"]), _p(keep), _p(dropped), _s())
    if int(dropped.item()) == 0:
        return rows
    idx, cnt = compact(keep)
    idx = idx[:int(cnt.item())]
    return {k: v.index_select(0, idx) for k, v in rows.items()}


def render_selected(scene, index, count, view, proj, campos, cam, bg, use_filter=True, stats=False):
    """Gather + activate the selected rows, drop the invalid ones as FilterGS.render does, and rasterize
    them (forward only, colours precomputed)."""
    n = int(count.item())                       # the host synchronisation for the row count
    rows = drop_invalid_rows(gather_activate(scene, index, count, campos, cap=n))
    e = torch.empty(0, device=scene.xyz.device)
    return _C.rasterize_gaussians(bg, rows["xyz"], rows["colors"], rows["opacity"], rows["scaling"],
                                  rows["rotation"], 1.0, e, view, proj, cam.tanfovx, cam.tanfovy, cam.H, cam.W, e, 0,
                                  campos, False, use_filter, False, 0.2, 0.2, 0.05, 0.7, stats)
