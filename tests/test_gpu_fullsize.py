"""GPU: the headline workload at its full size (2,000,000 Gaussians of the urban aerial
scene, SH 3, the benchmark's 1920x1080 cameras) against the reference's own CUDA build and
through properties that do not depend on size.

* the reference build, forward: num_rendered, radii, 2D means, depths, conics, colours,
  sorted keys, tile ranges, n_contrib, point_id, final T and the image bit for bit on two
  cameras (the preprocess writes out the reference build's multiply-add grouping, and the
  compositing arithmetic is the reference's);
* the reference build, backward (ref_compat): the screen-space, colour, opacity, mean and SH
  gradients within 1e-4 norm-relative of the mean of three reference runs.  The covariance,
  scale and rotation gradients are sums of many cancelling per-pixel terms that the
  reference adds with float atomics in arbitrary order (its own runs differ by 4e-4 to 9e-4
  norm-relative), so they are held to accuracy instead: against an FP64 evaluation of the
  same equations (the CPU oracle in FP64) they must be no further than 1.25 times the mean
  distance of three reference runs from it.  The reference's own runs scatter widely around
  that mean (six runs of the 2-view batch: rotations 1.16e-3 to 1.52e-3), and a 3-run mean
  moves by about 5%, so 1.25 keeps the check from failing on the reference's noise while a
  wrong term (errors of 1e-2 and more) still fails it.  A 2-view batched step's summed
  gradients are checked against the sums of the per-view gradients the same way;
* binning: num_rendered equals the sum of tiles touched; the sorted keys are non-decreasing
  (tile, then depth bits); the tile ranges partition [0, K) in tile order; n_contrib never
  exceeds its tile's range;
* determinism: two forwards and two backwards give the same bits;
* the long-tile band path gives the tile path's bits;
* the batched path (two cameras) gives the plain path's images and summed gradients."""
import numpy as np
import pytest
import torch

from _helpers import norm_rel, ours, ref_buffers

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
GRAD_NAMES = ["means2D", "colors", "opacity", "means3D", "cov3D", "sh", "scales", "rotations"]
# gradients that sum many cancelling per-pixel terms: the reference's own atomic summation
# order moves them by more than 1e-4 from run to run
ILL_CONDITIONED = ("cov3D", "scales", "rotations")
# ours against FP64, relative to the mean distance of three reference runs from FP64
ACCURACY_MARGIN = 1.25


@pytest.fixture(scope="module")
def _scene_pair():
    import bench
    return bench.make_scene(2_000_000, torch.device("cuda"))


@pytest.fixture(scope="module")
def full(_scene_pair):
    import bench
    return _scene_pair[1], bench.rank_cameras(2, 0)


@pytest.fixture(scope="module")
def full_np(_scene_pair):
    return _scene_pair[0]


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _fwd(mod, scene, c):
    bg = torch.zeros(3, device="cuda")
    e = torch.empty(0, device="cuda") if mod is ours else torch.Tensor([])
    return mod.rasterize_gaussians(bg, scene["means3D"], e, scene["opacities"], scene["scales"], scene["rotations"],
                                   1.0, e, _t(c.viewmatrix), _t(c.projmatrix), c.tanfovx, c.tanfovy, c.H, c.W,
                                   scene["shs"], 3, _t(c.campos), False, True, False, 0.2, 0.2, 0.05, 0.7, False)


def _bwd(scene, c, f, dL, mod=None):
    mod = mod or ours
    e = torch.empty(0, device="cuda") if mod is ours else torch.Tensor([])
    return mod.rasterize_gaussians_backward(torch.zeros(3, device="cuda"), scene["means3D"], f[5], e,
                                             scene["scales"], scene["rotations"], 1.0, e, _t(c.viewmatrix),
                                             _t(c.projmatrix), c.tanfovx, c.tanfovy, dL, scene["shs"], 3,
                                             _t(c.campos), f[6], f[0], f[7], f[8], False)


def test_fullsize_vs_reference_and_binning_properties(cuda, ref, full):
    scene, cams = full
    P = int(scene["means3D"].shape[0])
    for c in cams:
        mine = _fwd(ours, scene, c)
        theirs = _fwd(ref, scene, c)
        torch.cuda.synchronize()
        K = mine[0]
        assert K == theirs[0] and K > 1_000_000
        assert torch.equal(mine[5], theirs[5]), "radii"
        po = ours.preprocess_outputs(mine[6], P)
        rb = ref_buffers(theirs, P, c.W, c.H)
        vis = mine[5] > 0
        for k in ("means2D", "depths", "conic_opacity", "rgb", "tiles_touched"):
            assert torch.equal(po[k][vis], rb[k][vis]), k
        keys, vals = ours.sorted_pairs(mine[6], mine[7], P, K)
        assert torch.equal(keys, rb["keys"]) and torch.equal(vals, rb["vals"]), "sorted pairs"
        io = ours.image_outputs(mine[8], c.W, c.H)
        for k in ("ranges", "n_contrib", "final_T"):
            assert torch.equal(io[k], rb[k]), k
        assert torch.equal(mine[2], theirs[2]), "point_id"
        assert torch.equal(mine[3], theirs[3]), "point_weight_pixel"
        assert torch.equal(mine[1], theirs[1]), "image"
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


def _fp64_grads(scene_np, c, dL):
    """The reference's splat math in FP64 (CPU oracle, ref_compat backward) for one view."""
    from oracle import oracle as O
    import os
    O.set_threads(os.cpu_count() or 1)
    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    s64 = O.Scene(f64(scene_np["means3D"]), f64(scene_np["opacities"]), c.W, c.H, c.tanfovx, c.tanfovy,
                  f64(c.viewmatrix).reshape(-1), f64(c.projmatrix).reshape(-1), f64(c.campos), shs=f64(scene_np["shs"]),
                  sh_degree=3, scales=f64(scene_np["scales"]), rotations=f64(scene_np["rotations"]))
    of = O.forward(s64, dtype=np.float64)
    return O.backward(s64, of, dL.cpu().numpy().astype(np.float64), dtype=np.float64)


def _nr(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _grad_check(name, mine, refs, exact=None):
    """Well-conditioned gradients: mine within GRAD_TOL of the mean of the reference runs.
    Ill-conditioned sums: mine no further from the FP64 evaluation `exact` than 1.25 times the
    reference runs' mean distance from it."""
    m = sum(r.double() for r in refs) / len(refs)
    if name in ILL_CONDITIONED:
        ours = _nr(mine.cpu(), exact)
        theirs = float(np.mean([_nr(r.cpu(), exact) for r in refs]))
        assert ours <= ACCURACY_MARGIN * theirs, (name, ours, theirs)
        return ours
    d = norm_rel(mine, m)
    assert d <= GRAD_TOL, (name, d, GRAD_TOL)
    return d


def test_fullsize_gradients_vs_reference(cuda, ref, full, full_np):
    scene, cams = full
    for i, c in enumerate(cams):
        g = torch.Generator(device="cuda").manual_seed(40 + i)
        dL = torch.randn(3, c.H, c.W, device="cuda", generator=g)
        mine = _bwd(scene, c, _fwd(ours, scene, c), dL)
        rf = _fwd(ref, scene, c)
        runs = [_bwd(scene, c, rf, dL, ref) for _ in range(3)]
        torch.cuda.synchronize()
        x = _fp64_grads(full_np, c, dL)
        for j, n in enumerate(GRAD_NAMES):
            assert mine[j].shape == runs[0][j].shape, n
            _grad_check(n, mine[j], [r[j] for r in runs], x.get(n))
        del runs


def test_fullsize_batched_gradients_vs_reference(cuda, ref, full, full_np):
    """One 2-view batched step: the shared gradients against the sums of the reference's
    per-view gradients (means3D, opacity, SH, scales, rotations)."""
    from filtergs_b200.batched import BatchedRasterizer, Camera
    scene, cams = full
    bc = [Camera(c.W, c.H, c.tanfovx, c.tanfovy, _t(c.viewmatrix), _t(c.projmatrix), _t(c.campos)) for c in cams]
    br = BatchedRasterizer(scene["means3D"], scene["opacities"], scene["scales"], scene["rotations"], bc,
                           shs=scene["shs"], sh_degree=3, bg=torch.zeros(3, device="cuda"), graph=True)
    g = torch.Generator(device="cuda").manual_seed(44)
    dls = [torch.randn(3, c.H, c.W, device="cuda", generator=g) for c in cams]
    for v, d in enumerate(dls):
        br.dL[v].copy_(d)
    br.step()
    br.check()
    keys = {"means3D": 3, "opacity": 2, "sh": 5, "scales": 6, "rotations": 7}
    sums = [{k: torch.zeros_like(v) for k, v in br.grad.items()} for _ in range(3)]
    exact = {k: 0.0 for k in keys}
    for c, d in zip(cams, dls):
        rf = _fwd(ref, scene, c)
        for s in sums:
            r = _bwd(scene, c, rf, d, ref)
            for k, j in keys.items():
                s[k] += r[j].reshape(s[k].shape)
        x = _fp64_grads(full_np, c, d)
        for k in keys:
            exact[k] = exact[k] + np.asarray(x[k], np.float64).reshape(-1)
    torch.cuda.synchronize()
    for k in keys:
        _grad_check(k, br.grad[k], [s[k] for s in sums], exact[k])
