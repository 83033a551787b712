"""PyTorch-CPU FP32 restatement of the reference's splat math: forward and backward of one view.

TEST INFRASTRUCTURE / CPU BASELINE ONLY: used by the CPU tests and by bench.py's
cpu_baseline leg, always as a checker or a timed baseline, never by the product.

It restates the reference's own torch helpers where they exist --
LoG/model/geometry.py (build_rotation :4-25, computeCov3D :27-42, transformPoint4x3
:44-45, computeCov2D0 :89-128) and LoG/model/sh_utils.py (eval_sh_wobase :31-73,
SH2RGB :78) -- and writes the CUDA rasterizer's remaining steps as vectorised torch
ops: the OGFS radius (antialias/cuda_rasterizer/forward.cu:339-369), ndc2Pix and
getRect (auxiliary.h:41-56), duplicateWithKeys + the stable (tile, depth) sort +
identifyTileRanges (rasterizer_impl.cu:113-194, 430-445) and renderCUDA's front-to-back
compositing with its 1/255 skip and T < 1e-4 termination (forward.cu:406-567).  The
compositing of one tile is a [pixels, records] matrix: exclusive transmittance by a
cumulative product, the first terminating record found per pixel, the contributions
masked after it.  The backward is torch autograd through the same ops, so it
differentiates the forward as computed (the CUDA path's `consistent` mode).

Like the reference, rotations are used as given (the CUDA kernels do not normalise
them) and the 2D dilation is max(cov, 0.3) when use_filter is set.
"""
import math

import torch

C0 = 0.28209479177387814
C1 = 0.4886025119029199
C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
      1.445305721320277, -0.5900435899266435]
TILE = 16


def rotation_matrix(q):
    """build_rotation (geometry.py:4-25) without its normalisation: R[:, r, c]."""
    r, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = torch.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - r * z), 2 * (x * z + r * y),
        2 * (x * y + r * z), 1 - 2 * (x * x + z * z), 2 * (y * z - r * x),
        2 * (x * z - r * y), 2 * (y * z + r * x), 1 - 2 * (x * x + y * y)], 1)
    return R.view(-1, 3, 3)


def cov3d(scales, rots, mod=1.0):
    """computeCov3D (geometry.py:27-42): L = R S, Sigma = L L^T."""
    L = rotation_matrix(rots) * (mod * scales)[:, None, :]
    return L @ L.transpose(1, 2)


def eval_sh_wobase(dirs, sh, degree):
    """sh_utils.py:31-73 (without the DC term); sh [N, coeffs-1, 3]."""
    x, y, z = dirs[:, 0:1], dirs[:, 1:2], dirs[:, 2:3]
    result = -C1 * y * sh[:, 0] + C1 * z * sh[:, 1] - C1 * x * sh[:, 2]
    if degree > 1:
        xx, yy, zz = x * x, y * y, z * z
        xy, yz, xz = x * y, y * z, x * z
        result = (result + C2[0] * xy * sh[:, 3] + C2[1] * yz * sh[:, 4] + C2[2] * (2.0 * zz - xx - yy) * sh[:, 5] +
                  C2[3] * xz * sh[:, 6] + C2[4] * (xx - yy) * sh[:, 7])
        if degree > 2:
            result = (result + C3[0] * y * (3 * xx - yy) * sh[:, 8] + C3[1] * xy * z * sh[:, 9] +
                      C3[2] * y * (4 * zz - xx - yy) * sh[:, 10] + C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * sh[:, 11] +
                      C3[4] * x * (4 * zz - xx - yy) * sh[:, 12] + C3[5] * z * (xx - yy) * sh[:, 13] +
                      C3[6] * x * (xx - 3 * yy) * sh[:, 14])
    return result


def preprocess(means, scales, rots, opac, shs, degree, cam, use_filter=True, ogfs=(0.2, 0.2, 0.05, 0.7)):
    """Per-Gaussian screen-space state (forward.cu:266-401): dict of 2D mean, view depth, conic, opacity,
    colour, integer radius and tile rectangle.  Differentiable in the float inputs."""
    W, H = cam.W, cam.H
    view = torch.as_tensor(cam.viewmatrix, dtype=torch.float32)
    proj = torch.as_tensor(cam.projmatrix, dtype=torch.float32)
    tanx, tany = float(cam.tanfovx), float(cam.tanfovy)
    fx, fy = W / (2.0 * tanx), H / (2.0 * tany)
    ones = torch.ones_like(means[:, :1])
    hom = torch.cat([means, ones], 1) @ proj                       # transformPoint4x4 (column-major)
    p_w = 1.0 / (hom[:, 3] + 1e-7)
    t = means @ view[:3, :3] + view[3, :3]                           # transformPoint4x3 (geometry.py:44-45)
    tz = t[:, 2]
    limx, limy = 1.3 * tanx, 1.3 * tany
    tx = torch.clamp(t[:, 0] / tz, -limx, limx) * tz
    ty = torch.clamp(t[:, 1] / tz, -limy, limy) * tz
    zero = torch.zeros_like(tz)
    J = torch.stack([fx / tz, zero, -(fx * tx) / (tz * tz),
                     zero, fy / tz, -(fy * ty) / (tz * tz),
                     zero, zero, zero], 1).view(-1, 3, 3)            # computeCov2D0 (geometry.py:89-128)
    T = J @ view[:3, :3].t()
    cov = T @ cov3d(scales, rots) @ T.transpose(1, 2)
    a, b, c = cov[:, 0, 0], cov[:, 0, 1], cov[:, 1, 1]
    if use_filter:
        a, c = torch.clamp_min(a, 0.3), torch.clamp_min(c, 0.3)
    det = a * c - b * b
    det_inv = 1.0 / det
    conic = torch.stack([c * det_inv, -b * det_inv, a * det_inv], 1)
    o = torch.clamp_min(opac.reshape(-1), 1e-6)
    # OGFS radius (forward.cu:339-369), opacity-aware, with the 3-sigma bound
    eps_scale, eps_max, floor, ratio = ogfs
    eps_pix = 1.0 / 255.0
    lam_raw = 1.0 - (1.0 - eps_pix) ** (TILE * TILE)
    lam = min(max(eps_pix + eps_scale * (lam_raw - eps_pix), eps_pix), eps_max)
    with torch.no_grad():
        energy = torch.clamp_min(torch.log(o) - math.log(lam), floor)
        mid = 0.5 * (a + c)
        disc = torch.clamp_min(mid * mid - det, 0.0)
        lmax = torch.clamp_min(torch.maximum(mid + disc.sqrt(), mid - disc.sqrt()), 1e-6)
        base = 3.0 * lmax.sqrt()
        major = torch.maximum(torch.minimum((2.0 * energy * lmax).sqrt(), base), ratio * base)
        radius = torch.clamp_min(torch.ceil(major + 1.0), 1).to(torch.int64)
        px = ((hom[:, 0] * p_w).double() + 1.0) * W - 1.0          # ndc2Pix in double (auxiliary.h:41-44)
        py = ((hom[:, 1] * p_w).double() + 1.0) * H - 1.0
        xy0 = torch.stack([(px * 0.5).float(), (py * 0.5).float()], 1)
        gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
        rf = radius.float()
        x0 = ((xy0[:, 0] - rf) / TILE).to(torch.int64).clamp(0, gx)
        y0 = ((xy0[:, 1] - rf) / TILE).to(torch.int64).clamp(0, gy)
        x1 = ((xy0[:, 0] + rf + TILE - 1) / TILE).to(torch.int64).clamp(0, gx)
        y1 = ((xy0[:, 1] + rf + TILE - 1) / TILE).to(torch.int64).clamp(0, gy)
        visible = (tz > 0.2) & (det != 0) & ((x1 - x0) * (y1 - y0) > 0)
        radius = torch.where(visible, radius, torch.zeros_like(radius))
    # the 2D mean with a gradient path: ndc2Pix is affine in the projected point
    xy = torch.stack([((hom[:, 0] * p_w + 1.0) * W - 1.0) * 0.5, ((hom[:, 1] * p_w + 1.0) * H - 1.0) * 0.5], 1)
    xy = xy + (xy0 - xy).detach()                                    # the reference's bits, its gradient
    if shs is not None:
        d = means - torch.as_tensor(cam.campos, dtype=torch.float32)[None]
        d = d / torch.norm(d, dim=-1, keepdim=True)
        col = shs[:, 0] * C0 + 0.5
        if degree > 0:
            col = col + eval_sh_wobase(d, shs[:, 1:], degree)
        col = torch.clamp_min(col, 0.0)
    else:
        col = None
    return dict(xy=xy, depth=tz, conic=conic, opacity=o, rgb=col, radius=radius, visible=visible,
                rect=(x0, y0, x1, y1))


def bin_pairs(pre, W, H):
    """duplicateWithKeys + stable sort by (tile, depth) + identifyTileRanges: (sorted Gaussian ids, ranges)."""
    with torch.no_grad():
        gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
        vis = torch.nonzero(pre["visible"]).flatten()
        x0, y0, x1, y1 = (r[vis] for r in pre["rect"])
        w, h = x1 - x0, y1 - y0
        cnt = w * h
        # depth order first (stable), then the pairs of each Gaussian, then a stable sort by tile
        dkey = pre["depth"][vis].detach().contiguous().view(torch.int32).to(torch.int64)
        order = torch.sort(dkey, stable=True).indices
        vis, x0, y0, w, cnt = vis[order], x0[order], y0[order], w[order], cnt[order]
        gid = torch.repeat_interleave(vis, cnt)
        first = torch.cumsum(cnt, 0) - cnt
        k = torch.arange(int(cnt.sum()), dtype=torch.int64) - torch.repeat_interleave(first, cnt)
        ww = torch.repeat_interleave(w, cnt)
        tile = (torch.repeat_interleave(y0, cnt) + k // ww) * gx + torch.repeat_interleave(x0, cnt) + k % ww
        s = torch.sort(tile, stable=True)
        ids = gid[s.indices]
        counts = torch.bincount(s.values, minlength=gx * gy)
        ends = torch.cumsum(counts, 0)
        ranges = torch.stack([ends - counts, ends], 1)
    return ids, ranges


def render_tile(xy, con, op, rgb, t, W, H, bg):
    """renderCUDA (forward.cu:406-567) for tile t over its depth-ordered records (2D means, conics,
    opacities, colours): its pixels' colours [3, th, tw] and final transmittance."""
    gx = (W + TILE - 1) // TILE
    tx, ty = t % gx, t // gx
    xs = torch.arange(tx * TILE, min(W, tx * TILE + TILE), dtype=torch.float32)
    ys = torch.arange(ty * TILE, min(H, ty * TILE + TILE), dtype=torch.float32)
    pyy, pxx = torch.meshgrid(ys, xs, indexing="ij")
    pix = torch.stack([pxx.reshape(-1), pyy.reshape(-1)], 1)               # [n_pix, 2]
    d = xy[None, :, :] - pix[:, None, :]                                    # [n_pix, n, 2]
    dx, dy = d[..., 0], d[..., 1]
    power = -0.5 * (con[None, :, 0] * dx * dx + con[None, :, 2] * dy * dy) - con[None, :, 1] * dx * dy
    alpha = torch.clamp_max(op[None, :] * torch.exp(power), 0.99)
    valid = (power <= 0) & (alpha >= 1.0 / 255.0)
    a = torch.where(valid, alpha, torch.zeros_like(alpha))
    trans = torch.cumprod(1.0 - a, 1)                                      # T after each record
    with torch.no_grad():
        stop = valid & (trans < 1e-4)
        n = a.shape[1]
        idx = torch.arange(n)[None, :].expand_as(stop)
        first = torch.where(stop, idx, torch.full_like(idx, n)).min(1).values
        take = valid & (idx < first[:, None])
    a = torch.where(take, a, torch.zeros_like(a))
    trans = torch.cumprod(1.0 - a, 1)
    T_before = torch.cat([torch.ones_like(trans[:, :1]), trans[:, :-1]], 1)
    w = a * T_before
    color = w @ rgb + trans[:, -1:] * bg[None, :]
    th, tw = ys.numel(), xs.numel()
    return color.t().reshape(3, th, tw), trans[:, -1].reshape(th, tw)


def forward_backward(means, scales, rots, opac, shs, degree, cam, dL, tiles=None, bg=(0.0, 0.0, 0.0)):
    """One view's forward over `tiles` (all tiles when None) and the autograd backward of
    sum(image * dL) over them.  Returns (image [3,H,W] with unrendered tiles zero, grads dict)."""
    params = [p.detach().clone().requires_grad_(True) for p in (means, scales, rots, opac, shs)]
    means_, scales_, rots_, opac_, shs_ = params
    W, H = cam.W, cam.H
    pre = preprocess(means_, scales_, rots_, opac_, shs_, degree, cam)
    ids, ranges = bin_pairs(pre, W, H)
    bgt = torch.as_tensor(bg, dtype=torch.float32)
    gx = (W + TILE - 1) // TILE
    ntiles = ranges.shape[0]
    tiles = range(ntiles) if tiles is None else tiles
    img = torch.zeros(3, H, W)
    loss = torch.zeros(())
    tiles = list(tiles)
    # one gather of every sampled tile's records, split per tile (a split's backward is one concatenation)
    sizes = [int(ranges[t, 1] - ranges[t, 0]) for t in tiles]
    ids_all = torch.cat([ids[int(ranges[t, 0]):int(ranges[t, 1])] for t in tiles]) if tiles else ids[:0]
    recs = [torch.split(pre[k][ids_all], sizes) for k in ("xy", "conic", "opacity", "rgb")]
    for i, t in enumerate(tiles):
        tx, ty = t % gx, t // gx
        x0, y0 = tx * TILE, ty * TILE
        if sizes[i]:
            col, _ = render_tile(recs[0][i], recs[1][i], recs[2][i], recs[3][i], t, W, H, bgt)
        else:
            col = bgt[:, None, None].expand(3, min(H, y0 + TILE) - y0, min(W, x0 + TILE) - x0)
        img[:, y0:y0 + col.shape[1], x0:x0 + col.shape[2]] = col.detach()
        loss = loss + (col * dL[:, y0:y0 + col.shape[1], x0:x0 + col.shape[2]]).sum()
    if not tiles:
        # no tile rendered: a unit gradient on every screen-space output still runs the
        # per-Gaussian backward (what a timing of the preprocess alone needs)
        loss = sum(pre[k].sum() for k in ("xy", "conic", "opacity", "rgb"))
    if loss.requires_grad:
        loss.backward()
    names = ("means3D", "scales", "rotations", "opacities", "shs")
    grads = {n: (p.grad if p.grad is not None else torch.zeros_like(p)) for n, p in zip(names, params)}
    return img, grads, pre, ranges
