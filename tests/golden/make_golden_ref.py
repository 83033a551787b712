"""Generate golden fixtures from the reference's OWN CUDA build (oracle/_ref).

Run on a machine with a GPU and the reference build present:

    python tests/golden/make_golden_ref.py

Writes tests/golden/ref_*.npz: the inputs of each case and the reference's
outputs (the `_C` forward/backward of antialias/rasterize_points.cu and the
internal per-Gaussian, per-pixel and sorted-pair state read out of its opaque
buffers; the FilterGS compute_radius_v2 module's visibility mask, radius and
depth).  The CPU tests check the C oracle against these fixtures.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from _helpers import Case, ref_buffers, run_backward, run_forward  # noqa: E402
from filtergs_b200 import synthetic as S  # noqa: E402
from oracle import build_ref  # noqa: E402


def raster_case(name, P, W, H, seed, degree=3, **kw):
    ref = build_ref.load("ref_rasterizer_C")
    sc, cam = S.small_scene(P=P, seed=seed, W=W, H=H, degree=degree)
    case = Case(sc, cam, **kw)
    fwd = run_forward(ref, case, stats=True)
    torch.cuda.synchronize()
    K = fwd[0]
    rb = ref_buffers(fwd, P, W, H)
    g = torch.Generator().manual_seed(seed + 1)
    dL = torch.randn(3, H, W, generator=g).cuda()
    grads = run_backward(ref, case, fwd, dL)
    out = dict(
        means3D=sc["means3D"], scales=sc["scales"], rotations=sc["rotations"], opacities=sc["opacities"],
        shs=sc["shs"], sh_degree=degree, colors=case.colors if case.colors is not None else np.zeros((0, 3), np.float32),
        bg=case.bg, use_filter=int(case.use_filter), W=W, H=H, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy,
        viewmatrix=cam.viewmatrix, projmatrix=cam.projmatrix, campos=cam.campos, dL=dL.cpu().numpy(),
        num_rendered=K, color=fwd[1].cpu().numpy(), point_id=fwd[2].cpu().numpy(),
        point_weight_pixel=fwd[3].cpu().numpy(), point_weight=fwd[4].cpu().numpy(), radii=fwd[5].cpu().numpy(),
        stats=fwd[9].numpy())
    for k in ("depths", "means2D", "conic_opacity", "rgb", "tiles_touched", "final_T", "n_contrib", "ranges",
              "vals", "keys"):
        if k in rb:
            out["ref_" + k] = rb[k].cpu().numpy()
    for n, t in zip(["means2D", "colors", "opacity", "means3D", "cov3D", "sh", "scales", "rotations"], grads):
        out["grad_" + n] = t.cpu().numpy()
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **out)
    print(name, "K", K, "visible", int((out["radii"] > 0).sum()))


def lod_case(name, P, seed):
    v2 = build_ref.load("ref_compute_radius_v2")
    tr = S.lod_tree(P=P, seed=seed, roots=2, max_depth=6, half_extent=40.0)
    c = tr["xyz"][tr["roots"]].mean(0)
    cam = S.look_at_camera(c + np.array([20.0, -120.0, 70.0]), c, W=320, H=180, fx=1600.0 / 6)
    d = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(d)  # noqa: E731
    fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
    args = (t(tr["xyz"]), t(tr["log_scales"]), t(tr["rotations"]), t(cam.projmatrix), t(cam.viewmatrix),
            t(tr["node_index"]), t(tr["ancestor_path"]), float(fx), float(fy), float(cam.tanfovx),
            float(cam.tanfovy))
    mask, rad, dep = v2.compute_visibility_radius(*args, 0.1, 1.5, 700.0)
    scal = torch.exp(t(tr["log_scales"]))
    rot = torch.nn.functional.normalize(t(tr["rotations"]))
    r3 = v2.compute_radius(t(tr["xyz"]), scal, rot, t(cam.projmatrix), t(cam.viewmatrix), float(fx), float(fy),
                           float(cam.tanfovx), float(cam.tanfovy))
    torch.cuda.synchronize()
    out = dict(tr, W=cam.W, H=cam.H, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy, viewmatrix=cam.viewmatrix,
               projmatrix=cam.projmatrix, campos=cam.campos, fx=fx, fy=fy, padding=0.1, radius_max=1.5,
               radius_filter_threshold=700.0, mask=mask.cpu().numpy(), radius2d=rad.cpu().numpy(),
               depth=dep.cpu().numpy(), scales_act=scal.cpu().numpy(), rot_norm=rot.cpu().numpy(),
               radius_v2=r3.cpu().numpy())
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **out)
    print(name, "nodes", P, "kept", int(out["mask"].sum()))


if __name__ == "__main__":
    assert build_ref.load("ref_rasterizer_C") is not None, "reference build missing"
    raster_case("sh3_filter", P=1200, W=96, H=64, seed=2101)
    raster_case("colors_nofilter_ragged", P=900, W=90, H=52, seed=2102, degree=0, colors_precomp=True,
                use_filter=False, bg=(0.3, 0.1, 0.7))
    raster_case("sh1_dense", P=3000, W=64, H=64, seed=2103, degree=1)
    lod_case("lod_tree", P=6000, seed=2104)
