"""The allocation-free forward entry point (fgs_forward_noalloc) against the
regular forward (fgs_forward_preprocess + fgs_forward_render).

fgs_forward_noalloc serves callers that cannot allocate device memory while
they render -- a render thread that must not pay cudaMalloc's device-wide
synchronisation, a plugin whose host application owns all device memory, a
process under a fixed memory budget.  It keeps the rasterizer's scratch in a
32 MiB library-owned device array, so this test checks that two calls in a
row (which reuse that array and must clear what the previous call left) give
the regular entry point's outputs, and that work too large for the array is
refused with FGS_ERR_CAPACITY.  The test allocates its inputs and outputs
with torch; the entry point itself allocates nothing.

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from _helpers import ours, small_case
from filtergs_b200 import _lib
from filtergs_b200._C import _args, _ptr

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5


def _inputs(case):
    a = case.torch_inputs()
    e = torch.Tensor([])
    sh = a["sh"] if a["sh"].numel() else None
    args = _args(case.P, a["degree"], int(sh.shape[1]) if sh is not None else 0, case.cam.W, case.cam.H,
                 a["background"], a["means3D"], sh, a["colors"] if a["colors"].numel() else e, a["opacity"],
                 a["scales"], 1.0, a["rotations"], e, a["viewmatrix"], a["projmatrix"], a["campos"],
                 case.cam.tanfovx, case.cam.tanfovy, False, case.use_filter, *case.ogfs, False, 0.0)
    return a, args


def _noalloc(case):
    a, args = _inputs(case)
    H, W, P = case.cam.H, case.cam.W, case.P
    dev = torch.device("cuda")
    radii = torch.full((P,), -7, dtype=torch.int32, device=dev)
    color = torch.full((3, H, W), float("nan"), device=dev)
    pid = torch.full((H, W), -7, dtype=torch.int32, device=dev)
    pwp = torch.full((H, W), float("nan"), device=dev)
    pw = torch.full((P,), float("nan"), device=dev)
    K = C.c_longlong(-1)
    st = _lib.lib().fgs_forward_noalloc(C.byref(args), _ptr(radii), _ptr(color), _ptr(pid), _ptr(pwp), _ptr(pw),
                                        C.byref(K), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, int(K.value), radii, color, pid, pwp, pw


def _regular(case):
    a = case.torch_inputs()
    return ours.rasterize_gaussians(*a.values(), False, *case.ogfs, False)


def test_noalloc_matches_regular_forward_twice(cuda):
    # two different calls in a row: the second reuses the array the first left behind
    for case in (small_case(P=6000, seed=1101, W=256, H=192), small_case(P=3000, seed=1102, W=200, H=136)):
        st, K, radii, color, pid, pwp, pw = _noalloc(case)
        assert st == _lib.FGS_OK, _lib.status_string(st)
        ref = _regular(case)
        assert K == ref[0]
        assert torch.equal(radii, ref[5])
        assert torch.equal(pid, ref[2])
        assert (color - ref[1]).abs().max().item() <= IMG_TOL
        assert (pwp - ref[3]).abs().max().item() <= IMG_TOL
        assert (pw - ref[4]).abs().max().item() <= IMG_TOL


def test_noalloc_rejects_work_beyond_its_array(cuda):
    cap = int(_lib.lib().fgs_noalloc_capacity_bytes())
    assert cap == 32 << 20
    # per-Gaussian state alone exceeds the array: refused before any work
    big = small_case(P=600_000, seed=1103, W=64, H=64)
    st = _noalloc(big)[0]
    assert st == _lib.FGS_ERR_CAPACITY
    # a normal call still works afterwards
    _check_normal_call(small_case(P=2000, seed=1104, W=128, H=128))


def test_noalloc_rejects_pairs_beyond_its_array(cuda):
    # few but large Gaussians on a large image: the per-Gaussian and per-pixel state
    # fit, the tile/Gaussian pairs found by the preprocess do not
    case = small_case(P=20_000, seed=1105, W=1024, H=1024)
    case.scene = dict(case.scene, scales=(case.scene["scales"] * 8.0).astype(np.float32))
    st = _noalloc(case)[0]
    assert st == _lib.FGS_ERR_CAPACITY
    ref = _regular(case)
    assert ref[0] * 48 > int(_lib.lib().fgs_noalloc_capacity_bytes())
    _check_normal_call(small_case(P=2500, seed=1106, W=160, H=120))


def test_noalloc_rejects_statistics(cuda):
    case = small_case(P=500, seed=1107, W=64, H=64)
    a, args = _inputs(case)
    args.ogfs_enable_stats = 1
    dev = torch.device("cuda")
    outs = [torch.zeros(case.P, dtype=torch.int32, device=dev), torch.zeros(3, 64, 64, device=dev),
            torch.zeros(64, 64, dtype=torch.int32, device=dev), torch.zeros(64, 64, device=dev),
            torch.zeros(case.P, device=dev)]
    K = C.c_longlong(-1)
    st = _lib.lib().fgs_forward_noalloc(C.byref(args), *[_ptr(o) for o in outs], C.byref(K),
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.FGS_ERR_ARG


def _check_normal_call(ok):
    st, K, radii, color, pid, pwp, pw = _noalloc(ok)
    assert st == _lib.FGS_OK
    ref = _regular(ok)
    assert K == ref[0] and torch.equal(radii, ref[5])
    assert (color - ref[1]).abs().max().item() <= IMG_TOL
    assert np.isfinite(color.cpu().numpy()).all()
