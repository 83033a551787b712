"""GPU: the training-step pieces (filtergs_b200/train.py, csrc/train.cu) against plain
PyTorch FP32 restatements of LoG's own code -- the SSIM module of LoG/render/loss.py:6-44
with the 0.8 L1 + 0.2 (1 - SSIM) loss of renderer.py:260-273 (autograd for the
gradient), the Adam step of sparse_optimizer.py:41-78 with the activations of
activation.py chained by autograd -- and the batched step against the plain step."""
import math

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from _helpers import S, norm_rel
from filtergs_b200 import train as T
from filtergs_b200.batched import Camera

pytestmark = pytest.mark.gpu


def _window(channel=3, size=11, sigma=1.5):
    g = torch.tensor([math.exp(-(x - size // 2) ** 2 / float(2 * sigma ** 2)) for x in range(size)])
    g = g / g.sum()
    w = g[:, None].mm(g[None, :]).float()[None, None]
    return w.expand(channel, 1, size, size).contiguous()


def _torch_loss(preds, targets):
    """renderer.py:260-273 on stacked [B,3,H,W] images, SSIM with padding 0 (loss.py:26-44)."""
    x, y = torch.stack(preds), torch.stack(targets)
    w = _window().to(x.device)
    mu1, mu2 = F.conv2d(x, w, groups=3), F.conv2d(y, w, groups=3)
    s11 = F.conv2d(x * x, w, groups=3) - mu1 ** 2
    s22 = F.conv2d(y * y, w, groups=3) - mu2 ** 2
    s12 = F.conv2d(x * y, w, groups=3) - mu1 * mu2
    C1, C2 = 0.01 ** 2, 0.03 ** 2
    ssim = ((2 * mu1 * mu2 + C1) * (2 * s12 + C2)) / ((mu1 ** 2 + mu2 ** 2 + C1) * (s11 + s22 + C2))
    return 0.2 * (1.0 - ssim.mean()) + 0.8 * (x - y).abs().mean()


def test_loss_and_gradient_vs_torch(cuda):
    g = torch.Generator(device="cuda").manual_seed(3)
    W, H, B = 97, 83, 3
    preds = [torch.rand(3, H, W, device="cuda", generator=g) for _ in range(B)]
    targets = [(p + 0.1 * torch.randn(3, H, W, device="cuda", generator=g)).clamp(0, 1) for p in preds]
    loss = T.Loss([(W, H)] * B, "cuda")
    grads = [torch.empty_like(p) for p in preds]
    loss(preds, targets, grads)
    xs = [p.clone().requires_grad_(True) for p in preds]
    ref = _torch_loss(xs, targets)
    ref.backward()
    assert abs(loss.value() - ref.item()) <= 1e-5 * abs(ref.item())
    for a, x in zip(grads, xs):
        assert norm_rel(a, x.grad) <= 1e-4, norm_rel(a, x.grad)
    # the sums are re-zeroed per call: the same inputs give the same loss
    loss(preds, targets, grads)
    assert abs(loss.value() - ref.item()) <= 1e-5 * abs(ref.item())


def _torch_adam(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-15):
    """sparse_optimizer.py:41-78 for one tensor (in place)."""
    m.mul_(b1).add_(g, alpha=1 - b1)
    v.mul_(b2).addcmul_(g, g, value=1 - b2)
    step_size = lr / (1 - b1 ** t)
    denom = v.sqrt() / math.sqrt(1 - b2 ** t) + eps
    p.add_(-step_size * (m / denom))


def test_adam_step_vs_torch(cuda):
    rng = torch.Generator(device="cuda").manual_seed(11)
    P, M = 5000, 16
    raw = dict(xyz=torch.randn(P, 3, device="cuda", generator=rng),
               log_scale=torch.randn(P, 3, device="cuda", generator=rng) - 3,
               rot=torch.randn(P, 4, device="cuda", generator=rng),
               logit=torch.randn(P, 1, device="cuda", generator=rng),
               shs=0.1 * torch.randn(P, M, 3, device="cuda", generator=rng))
    st = T.TrainState(raw["xyz"], raw["log_scale"], raw["rot"], raw["logit"], raw["shs"])
    assert torch.allclose(st.scale, torch.exp(raw["log_scale"]))
    assert torch.allclose(st.opac, torch.sigmoid(raw["logit"]))
    assert torch.allclose(st.rot, F.normalize(raw["rot"]))
    # torch side: raw leaves, activations by autograd
    leaves = {k: v.clone().requires_grad_(True) for k, v in raw.items()}
    ms = {k: torch.zeros_like(v) for k, v in raw.items()}
    vs = {k: torch.zeros_like(v) for k, v in raw.items()}
    lrs = dict(xyz=T.DEFAULT_LR[0], shs=T.DEFAULT_LR[1], logit=T.DEFAULT_LR[2], log_scale=T.DEFAULT_LR[3],
               rot=T.DEFAULT_LR[4])
    for t in (1, 2):
        vis = torch.rand(P, device="cuda", generator=rng) < 0.6
        gm, gsh = torch.randn(P, 3, device="cuda", generator=rng), torch.randn(P, M, 3, device="cuda", generator=rng)
        go, gs = torch.randn(P, 1, device="cuda", generator=rng), torch.randn(P, 3, device="cuda", generator=rng)
        gr = torch.randn(P, 4, device="cuda", generator=rng)
        st.flag.copy_(vis.to(torch.uint8))
        st.adam(gm, gsh, go, gs, gr)
        for v in leaves.values():
            v.grad = None
        act = (leaves["xyz"] * gm).sum() + (leaves["shs"] * gsh).sum() + (torch.sigmoid(leaves["logit"]) * go).sum() \
            + (torch.exp(leaves["log_scale"]) * gs).sum() + (F.normalize(leaves["rot"]) * gr).sum()
        act.backward()
        with torch.no_grad():
            for k, leaf in leaves.items():
                p, gk, mk, vk = leaf.data[vis], leaf.grad[vis], ms[k][vis], vs[k][vis]
                _torch_adam(p, gk, mk, vk, t, lrs[k])
                leaf.data[vis], ms[k][vis], vs[k][vis] = p, mk, vk
    torch.cuda.synchronize()
    assert int(st.step.item()) == 2
    for mine, k in ((st.xyz, "xyz"), (st.shs, "shs"), (st.opac_logit, "logit"), (st.log_scale, "log_scale"),
                    (st.rot_raw, "rot")):
        assert torch.allclose(mine, leaves[k].data, rtol=1e-5, atol=1e-6), (k, (mine - leaves[k].data).abs().max())
    names = dict(xyz="xyz", shs="shs", opacity="logit", scale="log_scale", rotation="rot")
    for mine_key, k in names.items():
        # moments are differences of O(0.1) and O(1e-3) terms: absolute tolerance at their ulp scale
        assert torch.allclose(st.m[mine_key], ms[k], rtol=1e-5, atol=1e-7), mine_key
        assert torch.allclose(st.v[mine_key], vs[k], rtol=1e-5, atol=1e-9), mine_key
    assert torch.allclose(st.scale, torch.exp(st.log_scale)) and torch.allclose(st.opac, torch.sigmoid(st.opac_logit))


def _train_setup(P=60_000, nviews=3, seed=6001):
    sc = S.urban_scene(P=P, seed=seed, half_extent=120.0, buildings=40)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    logit = torch.logit(t(sc["opacities"]).clamp(1e-4, 1 - 1e-4))
    state_args = (t(sc["means3D"]), torch.log(t(sc["scales"])), t(sc["rotations"]), logit, t(sc["shs"]))
    rng = np.random.default_rng(seed + 1)
    cams = []
    for i in range(nviews):
        W, H = (320, 180) if i % 2 == 0 else (256, 144)
        c = S.aerial_camera(rng, W=W, H=H, fx=1600.0 * W / 1920, altitude=rng.uniform(60, 120),
                            pitch_deg=rng.uniform(35, 70), xy_range=50.0)
        cams.append(Camera(c.W, c.H, c.tanfovx, c.tanfovy, t(c.viewmatrix), t(c.projmatrix), t(c.campos)))
    # targets: renders of a perturbed copy
    g = torch.Generator(device="cuda").manual_seed(seed + 2)
    pert = T.TrainState(state_args[0] + 0.05 * torch.randn(P, 3, device="cuda", generator=g), *state_args[1:4],
                        state_args[4] + torch.cat([0.1 * torch.randn(P, 1, 3, device="cuda", generator=g),
                                                   torch.zeros(P, 15, 3, device="cuda")], 1))
    e = torch.empty(0, device="cuda")
    bg = torch.zeros(3, device="cuda")
    from filtergs_b200._C import rasterize_gaussians
    targets = [rasterize_gaussians(bg, pert.xyz, e, pert.opac, pert.scale, pert.rot, 1.0, e, c.viewmatrix,
                                   c.projmatrix, c.tanfovx, c.tanfovy, c.H, c.W, pert.shs, 3, c.campos, False, True,
                                   False, 0.2, 0.2, 0.05, 0.7, False)[1].clone() for c in cams]
    return state_args, cams, targets


@pytest.mark.parametrize("graph", [False, True])
def test_batched_step_equals_plain_step(cuda, graph):
    """Three views, three steps: the graph-captured batched step and the one-view-per-call step give
    bit-identical parameters, Adam moments and statistics (deterministic backward, same view order)."""
    state_args, cams, targets = _train_setup()
    a, b = T.TrainState(*state_args), T.TrainState(*state_args)
    bt = T.BatchedTrainer(a, cams, targets, graph=graph)
    pt = T.PlainTrainer(b, cams, targets)
    losses = []
    for _ in range(3):
        bt.step()
        pt.step()
        losses.append((bt.loss.value(), pt.loss.value()))
    bt.check()
    torch.cuda.synchronize()
    for x, y in zip(a.raw().values(), b.raw().values()):
        assert torch.equal(x, y)
    for k in a.m:
        assert torch.equal(a.m[k], b.m[k]) and torch.equal(a.v[k], b.v[k]), k
    assert torch.equal(a.grad_sum, b.grad_sum) and torch.equal(a.vis_count, b.vis_count)
    assert int(a.vis_count.max()) <= 9 and int((a.vis_count > 0).sum()) > 1000  # 3 views x 3 steps
    assert all(x == y for x, y in losses)
    assert losses[-1][0] < losses[0][0]   # the optimizer moves toward the targets
