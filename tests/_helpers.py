"""Shared helpers for the parity tests: scene construction, calls into this
library, into the reference build (oracle/_ref) and into the CPU oracle."""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from filtergs_b200 import _C as ours  # noqa: E402
from filtergs_b200 import synthetic as S  # noqa: E402
from oracle import build_ref  # noqa: E402
from oracle import oracle as O  # noqa: E402

OGFS_DEFAULT = (0.2, 0.2, 0.05, 0.7)


def ref_module():
    return build_ref.load("ref_rasterizer_C")


def ref_v2_module():
    return build_ref.load("ref_compute_radius_v2")


def ref_gather_module():
    return build_ref.load("ref_gather_attributes")


class Case:
    """One rasterizer call: numpy inputs + camera, convertible to torch/oracle form."""

    def __init__(self, scene, cam, use_filter=True, bg=(0.0, 0.0, 0.0), colors_precomp=False, cov3D_precomp=None,
                 ogfs=OGFS_DEFAULT, scale_modifier=1.0, filter3d=0.0):
        self.scene, self.cam = scene, cam
        self.use_filter, self.bg = use_filter, np.asarray(bg, np.float32)
        self.ogfs = ogfs
        self.scale_modifier = scale_modifier
        self.filter3d = filter3d
        self.colors = None
        if colors_precomp:
            rng = np.random.default_rng(7)
            self.colors = rng.uniform(0, 1, (scene["means3D"].shape[0], 3)).astype(np.float32)
        self.cov3D = cov3D_precomp

    @property
    def P(self):
        return self.scene["means3D"].shape[0]

    def torch_inputs(self, device="cuda"):
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        e = torch.Tensor([])
        sc = self.scene
        use_sr = self.cov3D is None
        return dict(
            background=t(self.bg), means3D=t(sc["means3D"]),
            colors=t(self.colors) if self.colors is not None else e,
            opacity=t(sc["opacities"]),
            scales=t(sc["scales"]) if use_sr else e, rotations=t(sc["rotations"]) if use_sr else e,
            scale_modifier=self.scale_modifier,
            cov3D_precomp=t(self.cov3D) if self.cov3D is not None else e,
            viewmatrix=t(self.cam.viewmatrix), projmatrix=t(self.cam.projmatrix),
            tan_fovx=self.cam.tanfovx, tan_fovy=self.cam.tanfovy, image_height=self.cam.H,
            image_width=self.cam.W, sh=t(sc["shs"]) if self.colors is None else e,
            degree=sc["sh_degree"] if self.colors is None else 0, campos=t(self.cam.campos),
            prefiltered=False, use_filter=self.use_filter)

    def oracle_scene(self):
        sc = self.scene
        use_sr = self.cov3D is None
        return O.Scene(sc["means3D"], sc["opacities"], self.cam.W, self.cam.H, self.cam.tanfovx, self.cam.tanfovy,
                       self.cam.viewmatrix.reshape(-1), self.cam.projmatrix.reshape(-1), self.cam.campos,
                       bg=self.bg, shs=sc["shs"] if self.colors is None else None,
                       sh_degree=sc["sh_degree"] if self.colors is None else 0, colors_precomp=self.colors,
                       scales=sc["scales"] if use_sr else None, rotations=sc["rotations"] if use_sr else None,
                       cov3D_precomp=self.cov3D, scale_modifier=self.scale_modifier, use_filter=self.use_filter,
                       ogfs=self.ogfs, filter3d=self.filter3d)


def run_forward(mod, case, stats=False, **extra):
    a = case.torch_inputs()
    return mod.rasterize_gaussians(*a.values(), False, *case.ogfs, stats, **extra)


def run_backward(mod, case, fwd, dL, **extra):
    a = case.torch_inputs()
    K, color, pid, pwp, pw, radii, geom, binning, img, stats = fwd
    return mod.rasterize_gaussians_backward(
        a["background"], a["means3D"], radii, a["colors"], a["scales"], a["rotations"], a["scale_modifier"],
        a["cov3D_precomp"], a["viewmatrix"], a["projmatrix"], a["tan_fovx"], a["tan_fovy"], dL, a["sh"],
        a["degree"], a["campos"], geom, K, binning, img, False, **extra)


def _a128(x):
    return (x + 127) & ~127


def ref_buffers(fwd, P, W, H):
    """Views into the reference's opaque buffers (rasterizer_impl.cu:211-250, 128-byte carving)."""
    K, geom, binning, img = fwd[0], fwd[6], fwd[7], fwd[8]
    N = W * H
    out = {}
    o = 0
    depths = geom[o:o + 4 * P].view(torch.float32)
    o = _a128(o + 4 * P)
    o = _a128(o + 3 * P)          # clamped
    o = _a128(o + 4 * P)          # internal radii
    means2D = geom[o:o + 8 * P].view(torch.float32).view(P, 2)
    o = _a128(o + 8 * P)
    o = _a128(o + 24 * P)         # cov3D
    conic = geom[o:o + 16 * P].view(torch.float32).view(P, 4)
    o = _a128(o + 16 * P)
    rgb = geom[o:o + 12 * P].view(torch.float32).view(P, 3)
    o = _a128(o + 12 * P)
    tiles = geom[o:o + 4 * P].view(torch.int32)
    out.update(depths=depths, means2D=means2D, conic_opacity=conic, rgb=rgb, tiles_touched=tiles)
    o = 0
    out["final_T"] = img[o:o + 4 * N].view(torch.float32)
    o = _a128(o + 4 * N)
    out["n_contrib"] = img[o:o + 4 * N].view(torch.int32)
    o = _a128(o + 4 * N)
    T = ((W + 15) // 16) * ((H + 15) // 16)
    out["ranges"] = img[o:o + 8 * T].view(torch.int32).view(T, 2)
    if K:
        o = 0
        out["vals"] = binning[o:o + 4 * K].view(torch.int32)
        o = _a128(o + 4 * K)
        o = _a128(o + 4 * K)
        out["keys"] = binning[o:o + 8 * K].view(torch.int64)
    return out


def norm_rel(a, b):
    a = a.double().reshape(-1)
    b = b.double().reshape(-1)
    d = torch.linalg.norm(a - b)
    n = torch.linalg.norm(b)
    return float(d / n) if n > 0 else float(d)


def small_case(P=10000, seed=1000, W=256, H=256, **kw):
    sc, cam = S.small_scene(P=P, seed=seed, W=W, H=H)
    return Case(sc, cam, **kw)
