"""GPU: the headline workload at its full size (2,000,000 Gaussians of the urban aerial
scene, SH 3, the benchmark's 1920x1080 cameras) checked through properties that do not
depend on size, and against the reference's own CUDA build.

* the reference build: num_rendered, radii, the 2D means and depths bit-exact.  The conic
  of a few percent of the visible Gaussians differs from the reference's by some ulps (the
  compilers fuse the covariance chain's multiply-adds differently), which moves the
  early-termination test T < 1e-4 of a handful of pixels per view and the colour of a few
  hundred: n_contrib and point_id are held to all but 1e-5 of the pixels (measured: 2-3 and
  0 of 2,073,600), image values to 1e-5 in all but 2e-4 of them (measured: 419 of 6.2 M
  values beyond it, the largest 2.9e-4);
* binning: num_rendered equals the sum of tiles touched; the sorted keys are non-decreasing
  (tile, then depth bits); the tile ranges partition [0, K) in tile order; n_contrib never
  exceeds its tile's range;
* determinism: two forwards and two backwards give the same bits;
* the long-tile band path gives the tile path's bits;
* the batched path (two cameras) gives the plain path's images and summed gradients."""
import numpy as np
import pytest
import torch

from _helpers import ours, ref_buffers

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
PIXEL_FRACTION = 1e-5


@pytest.fixture(scope="module")
def full():
    import bench
    sc, scene = bench.make_scene(2_000_000, torch.device("cuda"))
    cams = bench.rank_cameras(2, 0)
    return scene, cams


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _fwd(mod, scene, c):
    bg = torch.zeros(3, device="cuda")
    e = torch.empty(0, device="cuda") if mod is ours else torch.Tensor([])
    return mod.rasterize_gaussians(bg, scene["means3D"], e, scene["opacities"], scene["scales"], scene["rotations"],
                                   1.0, e, _t(c.viewmatrix), _t(c.projmatrix), c.tanfovx, c.tanfovy, c.H, c.W,
                                   scene["shs"], 3, _t(c.campos), False, True, False, 0.2, 0.2, 0.05, 0.7, False)


def _bwd(scene, c, f, dL):
    e = torch.empty(0, device="cuda")
    return ours.rasterize_gaussians_backward(torch.zeros(3, device="cuda"), scene["means3D"], f[5], e,
                                             scene["scales"], scene["rotations"], 1.0, e, _t(c.viewmatrix),
                                             _t(c.projmatrix), c.tanfovx, c.tanfovy, dL, scene["shs"], 3,
                                             _t(c.campos), f[6], f[0], f[7], f[8], False)


def test_fullsize_vs_reference_and_binning_properties(cuda, ref, full):
    scene, cams = full
    c = cams[0]
    P, N = int(scene["means3D"].shape[0]), c.W * c.H
    mine = _fwd(ours, scene, c)
    theirs = _fwd(ref, scene, c)
    torch.cuda.synchronize()
    K = mine[0]
    assert K == theirs[0] and K > 1_000_000
    assert torch.equal(mine[5], theirs[5]), "radii"
    po = ours.preprocess_outputs(mine[6], P)
    rb = ref_buffers(theirs, P, c.W, c.H)
    vis = mine[5] > 0
    assert torch.equal(po["means2D"][vis], rb["means2D"][vis]) and torch.equal(po["depths"][vis], rb["depths"][vis])
    io = ours.image_outputs(mine[8], c.W, c.H)
    assert int((io["n_contrib"] != rb["n_contrib"]).sum()) <= PIXEL_FRACTION * N, "n_contrib"
    assert int((mine[2] != theirs[2]).sum()) <= PIXEL_FRACTION * N, "point_id"
    d = (mine[1] - theirs[1]).abs()
    assert float(d.max()) <= 1e-3 and int((d > IMG_TOL).sum()) <= 2e-4 * 3 * N, "image"
    # binning properties
    assert int(po["tiles_touched"][vis].sum()) == K
    keys, _vals = ours.sorted_pairs(mine[6], mine[7], P, K)
    assert bool((keys[1:] >= keys[:-1]).all()), "sorted keys"
    r = io["ranges"].long()
    nonempty = r[:, 1] > r[:, 0]
    assert int((r[:, 1] - r[:, 0]).sum()) == K
    starts, ends = r[nonempty, 0], r[nonempty, 1]
    assert int(starts[0]) == 0 and int(ends[-1]) == K and torch.equal(starts[1:], ends[:-1])
    gx = (c.W + 15) // 16
    tile_of_pixel = (torch.arange(c.H, device="cuda")[:, None] // 16) * gx + torch.arange(c.W, device="cuda")[None] // 16
    assert bool((io["n_contrib"].long() <= (r[:, 1] - r[:, 0])[tile_of_pixel.reshape(-1)]).all())


def test_fullsize_determinism_and_band_path(cuda, full):
    from filtergs_b200 import _lib
    scene, cams = full
    c = cams[0]
    g = torch.Generator(device="cuda").manual_seed(21)
    dL = torch.randn(3, c.H, c.W, device="cuda", generator=g)
    split = _lib.get_render_split()
    try:
        _lib.set_render_split(0, 0)
        a = _fwd(ours, scene, c)
        b = _fwd(ours, scene, c)
        for i in (1, 2, 3, 4, 5):
            assert torch.equal(a[i], b[i]), i
        ga, gb = _bwd(scene, c, a, dL), _bwd(scene, c, b, dL)
        for x, y in zip(ga, gb):
            assert torch.equal(x, y)
        _lib.set_render_split(256, 3)
        s = _fwd(ours, scene, c)
        for i in (1, 2, 3, 4):
            assert torch.equal(a[i], s[i]), ("band path", i)
        for x, y in zip(ga, _bwd(scene, c, s, dL)):
            assert torch.equal(x, y)
    finally:
        _lib.set_render_split(*split)


def test_fullsize_batched_equals_plain(cuda, full):
    from filtergs_b200.batched import BatchedRasterizer, Camera
    scene, cams = full
    bc = [Camera(c.W, c.H, c.tanfovx, c.tanfovy, _t(c.viewmatrix), _t(c.projmatrix), _t(c.campos)) for c in cams]
    br = BatchedRasterizer(scene["means3D"], scene["opacities"], scene["scales"], scene["rotations"], bc,
                           shs=scene["shs"], sh_degree=3, bg=torch.zeros(3, device="cuda"), graph=True)
    g = torch.Generator(device="cuda").manual_seed(22)
    dls = [torch.randn(3, c.H, c.W, device="cuda", generator=g) for c in cams]
    for v, d in enumerate(dls):
        br.dL[v].copy_(d)
    br.step()
    br.check()
    torch.cuda.synchronize()
    sums = {k: torch.zeros_like(v) for k, v in br.grad.items()}
    for v, c in enumerate(cams):
        f = _fwd(ours, scene, c)
        assert torch.equal(br.images[v], f[1]), v
        gr = _bwd(scene, c, f, dls[v])
        sums["means3D"] += gr[3]
        sums["sh"] += gr[5]
        sums["opacity"] += gr[2]
    for k in ("means3D", "sh", "opacity"):
        assert torch.equal(br.grad[k], sums[k]), k
