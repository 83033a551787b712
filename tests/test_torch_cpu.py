"""CPU: the PyTorch-CPU FP32 restatement of the reference's splat math (oracle/torch_cpu.py, the
CPU baseline that bench.py times) against the C oracle on the CPU-runnable scene: the same
radii and tile ranges, images within 1e-5, and its autograd gradients within 1e-4
norm-relative of the oracle's `consistent` backward (the forward as computed, differentiated)."""
import numpy as np
import torch

from _helpers import O, S
from oracle import torch_cpu as TC


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a))


def test_torch_cpu_restatement_matches_oracle():
    sc, cam = S.small_scene(P=4000, seed=1000, W=160, H=128)
    dL = np.random.default_rng(3).standard_normal((3, cam.H, cam.W)).astype(np.float32)
    img, g, pre, ranges = TC.forward_backward(_t(sc["means3D"]), _t(sc["scales"]), _t(sc["rotations"]),
                                              _t(sc["opacities"]), _t(sc["shs"]), 3, cam, _t(dL))
    o_sc = O.Scene(sc["means3D"], sc["opacities"], cam.W, cam.H, cam.tanfovx, cam.tanfovy,
                   cam.viewmatrix.reshape(-1), cam.projmatrix.reshape(-1), cam.campos, shs=sc["shs"], sh_degree=3,
                   scales=sc["scales"], rotations=sc["rotations"])
    o = O.forward(o_sc)
    assert np.array_equal(pre["radius"].numpy(), o["pre"]["radii"])
    assert np.array_equal(ranges.numpy().astype(np.int64), o["ranges"].astype(np.int64).reshape(-1, 2))
    assert np.abs(img.numpy() - o["color"]).max() <= 1e-5
    ob = O.backward(o_sc, o, dL, consistent=True)
    for k, ok in (("means3D", "means3D"), ("scales", "scales"), ("rotations", "rotations"),
                  ("opacities", "opacity"), ("shs", "sh")):
        a, b = g[k].numpy().reshape(-1).astype(np.float64), np.asarray(ob[ok]).reshape(-1).astype(np.float64)
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b), k


def test_torch_cpu_tile_sample_equals_full_render_on_those_tiles():
    sc, cam = S.small_scene(P=2000, seed=1001, W=96, H=80)
    dL = torch.zeros(3, cam.H, cam.W)
    args = (_t(sc["means3D"]), _t(sc["scales"]), _t(sc["rotations"]), _t(sc["opacities"]), _t(sc["shs"]), 3, cam)
    full, *_ = TC.forward_backward(*args, dL)
    part, *_ = TC.forward_backward(*args, dL, tiles=[3, 7, 11])
    gx = (cam.W + 15) // 16
    for t in (3, 7, 11):
        y0, x0 = (t // gx) * 16, (t % gx) * 16
        assert torch.equal(part[:, y0:y0 + 16, x0:x0 + 16], full[:, y0:y0 + 16, x0:x0 + 16])
