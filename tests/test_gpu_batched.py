"""GPU: the batched multi-view path (fgs_batch_*, CUDA-graph replay) against the
plain one-view-per-call path.  Images and radii are bit-identical (same kernels,
same arithmetic), and so are the shared gradients and the sum of the per-view
gradients (the backward is deterministic)."""
import numpy as np
import pytest
import torch

from _helpers import S, norm_rel, ours
from filtergs_b200 import _lib
from filtergs_b200.batched import BatchedRasterizer, Camera

pytestmark = pytest.mark.gpu


def _scene(P=300_000, seed=5001):
    sc = S.urban_scene(P=P, seed=seed, half_extent=150.0, buildings=60)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return {k: (t(v) if isinstance(v, np.ndarray) else v) for k, v in sc.items()}


def _cams(n, seed=5002):
    rng = np.random.default_rng(seed)
    res = [(320, 180), (640, 360), (480, 272), (250, 170)]
    out = []
    for i in range(n):
        W, H = res[i % len(res)]
        c = S.aerial_camera(rng, W=W, H=H, fx=1600.0 * W / 1920, altitude=rng.uniform(60, 120),
                            pitch_deg=rng.uniform(30, 75), xy_range=60.0)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        out.append(Camera(c.W, c.H, c.tanfovx, c.tanfovy, t(c.viewmatrix), t(c.projmatrix), t(c.campos)))
    return out


def _plain(sc, cam, dL, bg):
    e = torch.empty(0, device="cuda")
    f = ours.rasterize_gaussians(bg, sc["means3D"], e, sc["opacities"], sc["scales"], sc["rotations"], 1.0, e,
                                 cam.viewmatrix, cam.projmatrix, cam.tanfovx, cam.tanfovy, cam.H, cam.W, sc["shs"], 3,
                                 cam.campos, False, True, False, 0.2, 0.2, 0.05, 0.7, False)
    g = ours.rasterize_gaussians_backward(bg, sc["means3D"], f[5], e, sc["scales"], sc["rotations"], 1.0, e,
                                          cam.viewmatrix, cam.projmatrix, cam.tanfovx, cam.tanfovy, dL, sc["shs"], 3,
                                          cam.campos, f[6], f[0], f[7], f[8], False)
    return f, g


@pytest.mark.parametrize("graph", [False, True])
def test_batched_matches_plain(cuda, graph):
    sc = _scene()
    cams = _cams(6)
    bg = torch.zeros(3, device="cuda")
    br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams, shs=sc["shs"],
                           sh_degree=3, bg=bg, graph=graph)
    gen = torch.Generator(device="cuda").manual_seed(7)
    for v in range(len(cams)):
        br.dL[v].copy_(torch.randn(br.dL[v].shape, device="cuda", generator=gen))
    for _ in range(2):                       # replay twice: state left by the first must not leak
        br.step()
    br.check()
    torch.cuda.synchronize()

    def plain_sums():
        sums = {k: torch.zeros_like(v) for k, v in br.grad.items()}
        for v, cam in enumerate(cams):
            f, g = _plain(sc, cam, br.dL[v], bg)
            assert torch.equal(br.radii[v], f[5]), v
            assert torch.equal(br.images[v], f[1]), v
            sums["means3D"] += g[3]
            sums["opacity"] += g[2]
            sums["sh"] += g[5]
            sums["scales"] += g[6]
            sums["rotations"] += g[7]
        return sums

    # The backward has no order-dependent float atomics (each Gaussian sums its per-pair
    # gradients in emission order, warps combine in a fixed order), so the batched sums
    # equal the per-view sums bit for bit.
    sums = plain_sums()
    for k in sums:
        assert torch.equal(br.grad[k], sums[k]), (k, norm_rel(br.grad[k], sums[k]))
    K = br.pair_counts()
    assert all(0 < k <= c for k, c in zip(K, br.capacity))


def test_batched_more_than_32_views(cuda):
    """34 views: the per-Gaussian backward walks two words of view bits; the shared gradients still
    equal the per-view sums (view order) bit for bit."""
    sc = _scene(P=100_000, seed=5021)
    cams = _cams(34, seed=5022)
    bg = torch.zeros(3, device="cuda")
    br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams, shs=sc["shs"],
                           sh_degree=3, bg=bg, graph=False)
    gen = torch.Generator(device="cuda").manual_seed(23)
    for v in range(len(cams)):
        br.dL[v].copy_(torch.randn(br.dL[v].shape, device="cuda", generator=gen))
    br.step()
    br.check()
    torch.cuda.synchronize()
    sums = {k: torch.zeros_like(v) for k, v in br.grad.items()}
    for v, cam in enumerate(cams):
        f, g = _plain(sc, cam, br.dL[v], bg)
        assert torch.equal(br.images[v], f[1]), v
        sums["means3D"] += g[3]
        sums["opacity"] += g[2]
        sums["sh"] += g[5]
        sums["scales"] += g[6]
        sums["rotations"] += g[7]
    for k in sums:
        assert torch.equal(br.grad[k], sums[k]), (k, norm_rel(br.grad[k], sums[k]))
    assert bool((sums["opacity"] != 0).any())


def test_batched_capacity_overflow_is_reported(cuda):
    sc = _scene(P=100_000, seed=5003)
    cams = _cams(2, seed=5004)
    br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams, shs=sc["shs"],
                           sh_degree=3, graph=False)
    br.capacity = [max(1, c // 4) for c in br.capacity]   # far too small
    br._build()
    br.forward()
    with pytest.raises(_lib.FgsError, match="too many"):
        br.check()
    br.replan()                                            # exact counts again
    br.forward()
    br.check()


def test_batched_set_io_retargets_captured_graph(cuda):
    """Swapping a view's image / gradient buffers after capture: the replay writes the new image
    buffer and reads the new gradient, with the same results as the original buffers."""
    sc = _scene(P=100_000, seed=5005)
    cams = _cams(3, seed=5006)
    br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams, shs=sc["shs"],
                           sh_degree=3, graph=True)
    gen = torch.Generator(device="cuda").manual_seed(9)
    for v in range(len(cams)):
        br.dL[v].copy_(torch.randn(br.dL[v].shape, device="cuda", generator=gen))
    br.step()
    br.check()
    img0 = [x.clone() for x in br.images]
    g0 = {k: v.clone() for k, v in br.grad.items()}
    old = list(br.images)
    new_img = [torch.full_like(x, -1.0) for x in br.images]
    new_dl = [2.0 * x for x in br.dL]
    br.set_io_many([0, 1, 2], new_img, new_dl)
    br.step()
    br.check()
    torch.cuda.synchronize()
    for v in range(3):
        assert torch.equal(new_img[v], img0[v]), v
        assert torch.equal(old[v], img0[v]), v          # the old buffers were not written again
    # the backward is linear in dL and scaling by 2 is exact in float: doubled upstream gradients
    # double every shared gradient exactly
    for k in g0:
        assert torch.equal(br.grad[k], 2.0 * g0[k]), k
    with pytest.raises(ValueError):
        br.set_io(0, torch.empty(3, 5, 5, device="cuda"))


def test_batched_long_tile_bands(cuda):
    """The multi-view forward with long tiles split into bands (a low threshold, so that most tiles
    of every view take the band path), at every band shape (16x2 and 8x4 take two records per
    step, 4x4 and 4x2 evaluate several records per step across lanes): images equal the unsplit
    batch's."""
    sc = _scene(P=200_000, seed=5011)
    cams = _cams(3, seed=5012)
    bg = torch.zeros(3, device="cuda")
    was = _lib.get_render_split()
    out = []
    try:
        for split, shape in ((0, 0), (64, 0), (64, 1), (64, 2), (64, 3)):
            _lib.set_render_split(split, shape)
            br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams,
                                   shs=sc["shs"], sh_degree=3, bg=bg, graph=False)
            br.forward()
            br.check()
            torch.cuda.synchronize()
            out.append([im.clone() for im in br.images])
            del br
    finally:
        _lib.set_render_split(*was)
    for shape_out in out[1:]:
        for x, y in zip(out[0], shape_out):
            assert torch.equal(x, y)


def test_batched_full_forward_outputs_match_plain(cuda):
    """With full_outputs the batched path also returns the reference call's point_id,
    point_weight_pixel and point_weight per view: equal to the plain path's, over two replays."""
    sc = _scene(P=200_000, seed=5011)
    cams = _cams(3, seed=5012)
    bg = torch.zeros(3, device="cuda")
    br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams, shs=sc["shs"],
                           sh_degree=3, bg=bg, graph=True, full_outputs=True)
    for _ in range(2):
        br.step()
    br.check()
    torch.cuda.synchronize()
    for v, cam in enumerate(cams):
        f, _ = _plain(sc, cam, br.dL[v], bg)
        assert torch.equal(br.images[v], f[1]), v
        assert torch.equal(br.point_id[v], f[2]), v
        assert torch.equal(br.point_weight_pixel[v], f[3]), v
        assert torch.equal(br.point_weight[v], f[4]), v


@pytest.mark.parametrize("graph", [False, True])
def test_step_events_overlap_copies(cuda, graph):
    """step(forward_done=, backward_ready=): the images are final when forward_done fires (a copy
    stream that waits for it reads the finished images while the backward runs), the backward waits
    for backward_ready (the upstream gradients written on another stream), and the results equal a
    plain step()'s."""
    sc = _scene(P=150_000, seed=5021)
    cams = _cams(3, seed=5022)
    bg = torch.zeros(3, device="cuda")
    br = BatchedRasterizer(sc["means3D"], sc["opacities"], sc["scales"], sc["rotations"], cams, shs=sc["shs"],
                           sh_degree=3, bg=bg, graph=graph)
    gen = torch.Generator(device="cuda").manual_seed(11)
    dls = [torch.randn(d.shape, device="cuda", generator=gen) for d in br.dL]
    for v, d in enumerate(dls):
        br.dL[v].copy_(d)
    br.step()
    br.check()
    torch.cuda.synchronize()
    want_img = [im.clone() for im in br.images]
    want_grad = {k: g.clone() for k, g in br.grad.items()}
    # the same step with the upstream gradients written on a side stream after the forward started
    for d in br.dL:
        d.zero_()
    side, copy = torch.cuda.Stream(), torch.cuda.Stream()
    fwd_done, dl_ready = torch.cuda.Event(), torch.cuda.Event()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for v, d in enumerate(dls):
            br.dL[v].copy_(d)
        dl_ready.record(side)
    br.step(forward_done=fwd_done, backward_ready=dl_ready)
    copy.wait_event(fwd_done)
    with torch.cuda.stream(copy):
        got_img = [im.clone() for im in br.images]
    torch.cuda.synchronize()
    br.check()
    assert fwd_done.query() and dl_ready.query()
    for x, y in zip(got_img, want_img):
        assert torch.equal(x, y)
    for k in want_grad:
        assert torch.equal(br.grad[k], want_grad[k]), k
