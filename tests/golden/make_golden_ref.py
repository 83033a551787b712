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


def urban_case(name="urban_1080", n=3000, out_dir=HERE):
    """The headline scene (2,000,000 Gaussians, 1920x1080 camera 0 of the benchmark) through the
    reference's forward; a seeded sample of n visible Gaussians with their inputs and the
    reference's per-Gaussian cov3D, conic and colour (for the CPU pin of oracle/ref_fp32.py)."""
    import bench
    ref = build_ref.load("ref_rasterizer_C")
    sc, scene = bench.make_scene(2_000_000, torch.device("cuda"))
    cam = bench.rank_cameras(1, 0)[0]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    bg, e = torch.zeros(3, device="cuda"), torch.Tensor([])
    fwd = ref.rasterize_gaussians(bg, scene["means3D"], e, scene["opacities"], scene["scales"], scene["rotations"],
                                  1.0, e, t(cam.viewmatrix), t(cam.projmatrix), cam.tanfovx, cam.tanfovy, cam.H, cam.W,
                                  scene["shs"], 3, t(cam.campos), False, True, False, 0.2, 0.2, 0.05, 0.7, False)
    torch.cuda.synchronize()
    P = 2_000_000
    rb = ref_buffers(fwd, P, cam.W, cam.H)
    geom, o = fwd[6], 0
    for nbytes in (4 * P, 3 * P, 4 * P, 8 * P):       # depths, clamped, internal radii, means2D
        o = (o + nbytes + 127) & ~127
    cov3D = geom[o:o + 24 * P].view(torch.float32).view(P, 6)
    radii = fwd[5].cpu().numpy()
    vis = np.nonzero(radii > 0)[0]
    pick = np.sort(np.random.default_rng(2105).choice(vis, size=n, replace=False))
    tp = torch.from_numpy(pick).cuda()
    out = dict(means3D=sc["means3D"][pick], scales=sc["scales"][pick], rotations=sc["rotations"][pick],
               opacities=sc["opacities"][pick], shs=sc["shs"][pick], sh_degree=3, colors=np.zeros((0, 3), np.float32),
               use_filter=1, W=cam.W, H=cam.H, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy,
               viewmatrix=cam.viewmatrix, projmatrix=cam.projmatrix, campos=cam.campos, radii=radii[pick],
               index=pick, ref_cov3D=cov3D[tp].cpu().numpy(), ref_conic_opacity=rb["conic_opacity"][tp].cpu().numpy(),
               ref_rgb=rb["rgb"][tp].cpu().numpy(), ref_means2D=rb["means2D"][tp].cpu().numpy(),
               ref_depths=rb["depths"][tp].cpu().numpy())
    np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), **out)
    print(name, "visible", len(vis), "sampled", n)


if __name__ == "__main__":
    assert build_ref.load("ref_rasterizer_C") is not None, "reference build missing"
    if sys.argv[1:2] == ["urban"]:                  # only the headline-scene sample, into the given directory
        urban_case(out_dir=sys.argv[2] if len(sys.argv) > 2 else HERE)
        sys.exit(0)
    raster_case("sh3_filter", P=1200, W=96, H=64, seed=2101)
    raster_case("colors_nofilter_ragged", P=900, W=90, H=52, seed=2102, degree=0, colors_precomp=True,
                use_filter=False, bg=(0.3, 0.1, 0.7))
    raster_case("sh1_dense", P=3000, W=64, H=64, seed=2103, degree=1)
    lod_case("lod_tree", P=6000, seed=2104)
    urban_case()
