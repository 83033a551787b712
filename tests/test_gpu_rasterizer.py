"""GPU parity of the rasterizer against the reference's own CUDA build
(oracle/_ref, bit-exact integers) and the CPU oracle (oracle/fgs_oracle.c).

Tolerances (from the build's contract): integer outputs -- radii, tiles,
sorted keys and ids, tile ranges, n_contrib, point_id -- bit-exact against the
reference build; images within 1e-5 absolute; gradients within 1e-4
norm-relative (backward_mode="ref_compat")."""
import numpy as np
import pytest
import torch

from _helpers import Case, O, S, norm_rel, ours, ref_buffers, run_backward, run_forward, small_case

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_TOL = 1e-4


def _cases():
    return {
        "sh3_filter": small_case(),
        "sh3_nofilter": small_case(seed=1010, use_filter=False),
        "colors_bg": small_case(P=6000, seed=1011, colors_precomp=True, bg=(0.2, 0.5, 0.9)),
        "ragged_250x170": small_case(P=5000, seed=1012, W=250, H=170),
    }


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_forward_bitexact_vs_reference(cuda, ref, name):
    case = _cases()[name]
    mine = run_forward(ours, case)
    theirs = run_forward(ref, case)
    torch.cuda.synchronize()
    P, W, H = case.P, case.cam.W, case.cam.H
    assert mine[0] == theirs[0], "num_rendered"
    assert torch.equal(mine[5], theirs[5]), "radii"
    rb = ref_buffers(theirs, P, W, H)
    po = ours.preprocess_outputs(mine[6], P)
    vis = mine[5] > 0
    assert torch.equal(po["tiles_touched"][vis], rb["tiles_touched"][vis])
    assert torch.equal(po["means2D"][vis], rb["means2D"][vis])
    assert torch.equal(po["depths"][vis], rb["depths"][vis])
    # the conic and the SH colour are float intermediates; the preprocess writes out the
    # reference build's multiply-add grouping, so they are equal bit for bit too
    assert torch.equal(po["conic_opacity"][vis], rb["conic_opacity"][vis]), "conic, opacity"
    if case.colors is None:
        assert torch.equal(po["rgb"][vis], rb["rgb"][vis]), "rgb"
    keys, vals = ours.sorted_pairs(mine[6], mine[7], P, mine[0])
    assert torch.equal(keys, rb["keys"]), "sorted keys"
    assert torch.equal(vals, rb["vals"]), "sorted point list"
    io = ours.image_outputs(mine[8], W, H)
    assert torch.equal(io["ranges"], rb["ranges"]), "tile ranges"
    assert torch.equal(io["n_contrib"], rb["n_contrib"]), "n_contrib"
    assert torch.equal(mine[2], theirs[2]), "point_id"
    assert torch.equal(io["final_T"], rb["final_T"]), "final T"
    assert torch.equal(mine[3], theirs[3]), "point_weight_pixel"
    if not case.bg.any():
        assert torch.equal(mine[1], theirs[1]), "image"
    assert (mine[1] - theirs[1]).abs().max().item() <= IMG_TOL, "image"
    # per-Gaussian max weight: exact max here, the reference's racy max is <= it
    assert bool((mine[4] >= theirs[4] - 1e-7).all())


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_backward_vs_reference(cuda, ref, name):
    case = _cases()[name]
    g = torch.Generator().manual_seed(5)
    dL = torch.randn(3, case.cam.H, case.cam.W, generator=g).cuda()
    mine = run_backward(ours, case, run_forward(ours, case), dL)
    theirs = run_backward(ref, case, run_forward(ref, case), dL)
    names = ["means2D", "colors", "opacity", "means3D", "cov3D", "sh", "scales", "rotations"]
    for n, a, b in zip(names, mine, theirs):
        assert a.shape == b.shape, n
        if b.numel() == 0:
            continue
        if b.abs().max() == 0:
            assert a.abs().max().item() == 0.0, n
            continue
        assert norm_rel(a, b) <= GRAD_TOL, (n, norm_rel(a, b))


def test_backward_is_deterministic(cuda):
    """Two backward passes over the same forward give bit-identical gradients: per-pair
    gradients are written once at their emission index and summed per Gaussian in a fixed
    order, so no float atomic decides a rounding."""
    case = small_case(P=20000, seed=1030, W=320, H=240)
    g = torch.Generator().manual_seed(9)
    dL = torch.randn(3, case.cam.H, case.cam.W, generator=g).cuda()
    fwd = run_forward(ours, case)
    a = run_backward(ours, case, fwd, dL)
    b = run_backward(ours, case, fwd, dL)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_forward_vs_oracle(cuda):
    case = small_case()
    mine = run_forward(ours, case)
    o = O.forward(case.oracle_scene())
    radii = mine[5].cpu().numpy()
    assert (radii != o["pre"]["radii"]).mean() <= 1e-3
    if np.array_equal(radii, o["pre"]["radii"]):
        keys, vals = ours.sorted_pairs(mine[6], mine[7], case.P, mine[0])
        assert np.array_equal(vals.cpu().numpy().astype(np.uint32), o["vals"])
    img = mine[1].cpu().numpy()
    assert np.abs(img - o["color"]).max() <= 1e-4
    assert np.mean(np.abs(img - o["color"]) > IMG_TOL) <= 1e-3


def test_backward_vs_oracle(cuda):
    case = small_case(P=4000, seed=1020)
    rng = np.random.default_rng(3)
    dL = rng.standard_normal((3, case.cam.H, case.cam.W)).astype(np.float32)
    fwd = run_forward(ours, case)
    mine = run_backward(ours, case, fwd, torch.from_numpy(dL).cuda())
    sc = case.oracle_scene()
    of = O.forward(sc)
    ob = O.backward(sc, of, dL)
    for n, a in zip(["means2D", "colors", "opacity", "means3D", "cov3D", "sh", "scales", "rotations"], mine):
        assert norm_rel(a.cpu(), torch.from_numpy(ob[n]).reshape(a.shape)) <= 1e-3, n


def test_stats_vs_reference(cuda, ref):
    case = small_case(P=8000, seed=1030)
    mine = run_forward(ours, case, stats=True)
    theirs = run_forward(ref, case, stats=True)
    a, b = mine[9], theirs[9]
    assert a.shape == b.shape
    assert torch.equal(a[1:6], b[1:6])          # averages, K, tiles, P
    assert a[8] == b[8] and torch.equal(a[9:9 + 64], b[9:9 + 64])  # bin count, edges
    assert abs(float(a[0] - b[0])) <= 1e-6 * max(1.0, abs(float(b[0])))  # bar_g (float sums)
    tot = float(b[6] + b[7])
    assert abs(float(a[6] - b[6])) <= 1e-3 * tot and abs(float(a[7] - b[7])) <= 1e-3 * tot
    T = (a.numel() - 9 - 128) // 2
    assert torch.equal(a[9 + 128 + T:], b[9 + 128 + T:])  # per-tile pair counts


def test_empty_and_culled(cuda, ref):
    case = small_case(P=100, seed=1040)
    case.scene["means3D"][:, 2] = -5.0      # everything behind the near plane
    mine = run_forward(ours, case)
    theirs = run_forward(ref, case)
    assert mine[0] == theirs[0] == 0
    assert torch.equal(mine[5], theirs[5])
    assert torch.equal(mine[1], theirs[1])
    assert torch.equal(mine[2], theirs[2])
    dL = torch.ones(3, case.cam.H, case.cam.W, device="cuda")
    for a, b in zip(run_backward(ours, case, mine, dL), run_backward(ref, case, theirs, dL)):
        assert torch.equal(a, b)
    z = ours.rasterize_gaussians(*Case(S.small_scene(P=1)[0], S.identity_camera()).torch_inputs().values())
    assert z[0] >= 0


def test_forward_4k_bitexact_vs_reference(cuda, ref):
    """A 3840x2160 view (32,400 tiles: 15-bit tile ids, the second tile-sort digit well used):
    count, radii, sorted keys and point list, ranges, n_contrib, point_id and the image equal the
    reference build's, and the well-conditioned gradients (2D means, colours, opacity, 3D means,
    SH) agree within the gradient tolerance (at this size the covariance, scale and rotation
    sums move with the order of the reference's float atomics, as at the headline size)."""
    case = small_case(P=120_000, seed=1045, W=3840, H=2160)
    mine = run_forward(ours, case)
    theirs = run_forward(ref, case)
    torch.cuda.synchronize()
    P, W, H = case.P, case.cam.W, case.cam.H
    assert mine[0] == theirs[0] and mine[0] > 1_000_000, "num_rendered"
    assert torch.equal(mine[5], theirs[5]), "radii"
    rb = ref_buffers(theirs, P, W, H)
    keys, vals = ours.sorted_pairs(mine[6], mine[7], P, mine[0])
    assert torch.equal(keys, rb["keys"]) and torch.equal(vals, rb["vals"]), "sorted pairs"
    io = ours.image_outputs(mine[8], W, H)
    assert torch.equal(io["ranges"], rb["ranges"]) and torch.equal(io["n_contrib"], rb["n_contrib"])
    assert torch.equal(mine[2], theirs[2]), "point_id"
    assert torch.equal(mine[1], theirs[1]), "image"
    g = torch.Generator().manual_seed(6)
    dL = torch.randn(3, H, W, generator=g).cuda()
    ga, gb = run_backward(ours, case, mine, dL), run_backward(ref, case, theirs, dL)
    for i in (0, 1, 2, 3, 5):   # means2D, colors, opacity, means3D, sh
        assert norm_rel(ga[i], gb[i]) <= GRAD_TOL, i


def test_zero_gaussians(cuda):
    case = small_case(P=10)
    a = case.torch_inputs()
    a["means3D"] = a["means3D"][:0]
    out = ours.rasterize_gaussians(*a.values())
    assert out[0] == 0 and out[1].abs().max() == 0 and out[5].numel() == 0


def test_mark_visible_and_radius_vs_reference(cuda, ref):
    case = small_case(P=5000, seed=1050)
    a = case.torch_inputs()
    a["means3D"][:500, 2] = 0.1
    assert torch.equal(ours.mark_visible(a["means3D"], a["viewmatrix"], a["projmatrix"]),
                       ref.mark_visible(a["means3D"], a["viewmatrix"], a["projmatrix"]))
    args = (a["means3D"], a["scales"], a["rotations"], a["viewmatrix"], a["projmatrix"], a["tan_fovx"],
            a["tan_fovy"], a["image_height"], a["image_width"])
    assert torch.equal(ours.compute_radius(*args), ref.compute_radius(*args))


def test_cov3d_precomp_and_filter3d(cuda, ref):
    """3D filter: the in-kernel filter equals feeding the reference the filtered covariance.  The
    covariance fed to the reference is cov3D + (0.2 z / fx)^2 on the diagonal, with cov3D and the
    view depth z in the reference build's own FP32 arithmetic (oracle/ref_fp32.py) and the filter
    terms as separately rounded float ops -- the same bits the fused kernel computes."""
    from oracle import ref_fp32 as R
    base = small_case(P=6000, seed=1060)
    sc, cam = base.scene, base.cam
    cov = R.cov3d(sc["scales"], sc["rotations"])
    z = R.view_z(sc["means3D"], cam.viewmatrix)
    fx = np.float32(cam.W) / (np.float32(2) * np.float32(cam.tanfovx))
    sf = (np.float32(0.2) * z) / fx
    v = (sf * sf).astype(np.float32)
    for k in (0, 3, 5):
        cov[:, k] = cov[:, k] + v
    pre = Case(sc, cam, cov3D_precomp=cov.astype(np.float32))
    mine = run_forward(ours, pre)
    theirs = run_forward(ref, pre)
    fused = run_forward(ours, base, filter3d_scale=0.2)
    torch.cuda.synchronize()
    assert mine[0] == theirs[0] == fused[0]
    for out in (mine, fused):
        assert torch.equal(out[5], theirs[5]), "radii"
        assert torch.equal(out[2], theirs[2]), "point_id"
        assert torch.equal(out[1], theirs[1]), "image"
    # the filter changed the render: it is not the unfiltered image
    plain = run_forward(ours, base)
    assert not torch.equal(plain[1], fused[1])


def test_autograd_module(cuda):
    from filtergs_b200.diff_gaussian_rasterization_wodilate import (GaussianRasterizationSettings,
                                                                    GaussianRasterizer)
    case = small_case(P=3000, seed=1070)
    a = case.torch_inputs()
    rs = GaussianRasterizationSettings(case.cam.H, case.cam.W, case.cam.tanfovx, case.cam.tanfovy, a["background"],
                                       1.0, a["viewmatrix"], a["projmatrix"], 3, a["campos"], False, False)
    r = GaussianRasterizer(rs)
    means = a["means3D"].clone().requires_grad_(True)
    means2D = torch.zeros_like(means, requires_grad=True)
    shs = a["sh"].clone().requires_grad_(True)
    op = a["opacity"].clone().requires_grad_(True)
    sc = a["scales"].clone().requires_grad_(True)
    rot = a["rotations"].clone().requires_grad_(True)
    color, radii, pid, pwp, pw = r(means, means2D, op, shs=shs, scales=sc, rotations=rot)
    (color.square().sum()).backward()
    for t in (means, means2D, shs, op, sc, rot):
        assert t.grad is not None and torch.isfinite(t.grad).all()
    assert r.latest_stats is not None and r.latest_stats["num_tiles"] == 256
    assert "tile_ratio" in r.latest_stats


def _dense_case():
    """40,000 small splats squeezed into a few tiles around the image centre (thousands of records
    per tile, like a distant LoD level)."""
    sc, cam = S.small_scene(P=40000, seed=1040, W=256, H=192)
    sc["means3D"][:, :2] *= 0.15
    return Case(sc, cam)


@pytest.mark.parametrize("stats,shape", [(False, 0), (True, 0), (False, 1), (False, 2), (True, 3)])
def test_long_tile_bands_equal_tile_path(cuda, ref, stats, shape):
    """Tiles with >= split_min records rendered in bands (one warp each; 16x2, 8x4, 4x4 or 4x2
    pixels) give exactly the outputs of the one-CTA-per-tile path, and the reference's integer
    outputs."""
    from filtergs_b200 import _lib
    case = _dense_case()
    W, H = case.cam.W, case.cam.H
    was = _lib.get_render_split()
    try:
        _lib.set_render_split(0, 0)
        a = run_forward(ours, case, stats=stats)
        _lib.set_render_split(512, shape)
        b = run_forward(ours, case, stats=stats)
    finally:
        _lib.set_render_split(*was)
    ia, ib = ours.image_outputs(a[8], W, H), ours.image_outputs(b[8], W, H)
    n = ia["ranges"][:, 1] - ia["ranges"][:, 0]
    assert int((n >= 512).sum()) >= 4 and int(n.max()) >= 4000
    for i, name in ((1, "color"), (2, "point_id"), (3, "point_weight_pixel"), (4, "point_weight")):
        assert torch.equal(a[i], b[i]), name
    assert torch.equal(ia["n_contrib"], ib["n_contrib"]) and torch.equal(ia["final_T"], ib["final_T"])
    if stats:
        # per-pair sums: band warps add with atomics, in another order than the tile path
        sa, sb = a[9].numpy(), b[9].numpy()
        assert np.allclose(sa, sb, rtol=1e-4, atol=1e-6)
    theirs = run_forward(ref, case, stats=False)
    rb = ref_buffers(theirs, case.P, W, H)
    assert torch.equal(ib["n_contrib"], rb["n_contrib"]), "n_contrib"
    assert torch.equal(b[2], theirs[2]), "point_id"
    assert (b[1] - theirs[1]).abs().max().item() <= IMG_TOL


def test_forward_identical_across_launch_shapes(cuda):
    """Every launch shape of the compositing kernel (pixels per thread, batch) and the band path
    give the same bits: the per-pixel arithmetic is written with explicit rounding."""
    from filtergs_b200 import _lib
    case = _dense_case()
    cfg, split = _lib.get_render_config(), _lib.get_render_split()
    outs = []
    try:
        for ppt, batch, sp in ((1, 64, (0, 0)), (2, 128, (0, 0)), (4, 256, (0, 0)), (2, 64, (256, 2)),
                               (1, 128, (256, 3))):
            _lib.set_render_config(ppt, batch, *cfg[2:4])
            _lib.set_render_split(*sp)
            outs.append(run_forward(ours, case))
    finally:
        _lib.set_render_config(*cfg)
        _lib.set_render_split(*split)
    for o in outs[1:]:
        for i in (1, 2, 3, 4):
            assert torch.equal(o[i], outs[0][i]), i


def test_backward_launch_shapes_agree(cuda, ref):
    """The backward at every pixels-per-thread shape and batch: the same gradients up to the order
    in which a thread adds its pixels' terms (each shape is deterministic), all within the
    reference tolerance."""
    from filtergs_b200 import _lib
    case = small_case(P=20000, seed=1040, W=320, H=240)
    g = torch.Generator().manual_seed(11)
    dL = torch.randn(3, case.cam.H, case.cam.W, generator=g).cuda()
    theirs = run_backward(ref, case, run_forward(ref, case), dL)
    fwd = run_forward(ours, case)
    cfg = _lib.get_render_config()
    grads = []
    try:
        for ppt, batch in ((1, 256), (2, 128), (4, 64), (4, 256)):
            _lib.set_render_config(cfg[0], cfg[1], ppt, batch)
            a = run_backward(ours, case, fwd, dL)
            b = run_backward(ours, case, fwd, dL)
            for x, y in zip(a, b):
                assert torch.equal(x, y), (ppt, batch)
            grads.append(a)
    finally:
        _lib.set_render_config(*cfg)
    names = ["means2D", "colors", "opacity", "means3D", "cov3D", "sh", "scales", "rotations"]
    for gr in grads:
        for n, x, y, t in zip(names, gr, grads[0], theirs):
            if t.numel() == 0 or t.abs().max() == 0:
                continue
            assert norm_rel(x, y) <= 1e-5, (n, norm_rel(x, y))
            assert norm_rel(x, t) <= GRAD_TOL, (n, norm_rel(x, t))
