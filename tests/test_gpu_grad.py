"""GPU: the CUDA backward in `consistent` mode against FP64 central differences
of the FP64 oracle forward on the small-scene workload (10,000 Gaussians, SH 3,
256x256, 2D filter on), 64 randomly chosen parameters.  FP32 gradients are
compared with relative error against max(|fd|, 1% of the RMS of all checked
differences); parameters straddling a discontinuity of the piecewise-smooth
renderer (the two step sizes disagree) are excluded and counted."""
import numpy as np
import pytest
import torch

from _fd import fd, pick_params
from _helpers import S, ours, run_backward, run_forward, small_case

pytestmark = pytest.mark.gpu

NAMES = {"means3D": 3, "scales": 6, "rotations": 7, "opacities": 2, "shs": 5}  # index in the gradient tuple


def test_consistent_backward_vs_fp64_central_differences(cuda):
    case = small_case(P=10000, seed=1000)
    sc, cam = case.scene, case.cam
    rng = np.random.default_rng(4101)
    dL = rng.standard_normal((3, cam.H, cam.W)).astype(np.float32)
    fwd = run_forward(ours, case)
    grads = run_backward(ours, case, fwd, torch.from_numpy(dL).cuda(), backward_mode="consistent")
    params = pick_params(sc, fwd[5].cpu().numpy(), 64, seed=4102)
    res = fd(sc, cam, dL.astype(np.float64), params)
    scale = np.sqrt(np.mean([r[0] ** 2 for r in res])) + 1e-12
    errs = []
    for (f, i, comp), (num, smooth) in zip(params, res):
        if not smooth:
            continue
        g = grads[NAMES[f]].detach().cpu().numpy()
        g = g.reshape((g.shape[0],) + sc[f].shape[1:])
        ana = float(g[(i,) + comp])
        errs.append(abs(ana - num) / max(abs(num), 1e-2 * scale))
    errs = np.array(errs)
    print(f"FD check: {len(errs)}/64 smooth parameters, median rel err {np.median(errs):.2e}, "
          f"max {errs.max():.2e}")
    assert len(errs) >= 56
    assert np.median(errs) <= 1e-4
    assert np.mean(errs <= 1e-3) >= 0.9


def test_ref_compat_and_consistent_differ_only_by_the_dilation_terms(cuda):
    # no 2D filter clamp active anywhere (large Gaussians): the modes differ only by +0.3 vs none
    case = small_case(P=2000, seed=4103, use_filter=False)
    case.scene["scales"] = case.scene["scales"] * 4
    dL = torch.randn(3, case.cam.H, case.cam.W, generator=torch.Generator().manual_seed(1)).cuda()
    f = run_forward(ours, case)
    a = run_backward(ours, case, f, dL, backward_mode="ref_compat")
    b = run_backward(ours, case, f, dL, backward_mode="consistent")
    # colour / opacity gradients do not depend on the dilation
    assert torch.allclose(a[1], b[1], rtol=1e-3, atol=1e-6)
    assert not torch.allclose(a[4], b[4], rtol=1e-3, atol=1e-6)
