"""GPU failure paths that fault nothing.

* A bounded look-back wait that runs out: a test hook makes one chunk of the first
  depth-sort pass keep its counts to itself, so the chunks after it wait on a status
  word that nothing sets.  With a short limit they give up, the forward reports
  FGS_ERR_TIMEOUT, and the next forward on the same context (hook off) gives the
  same bits as one run before the hook.
* prefiltered=True with a Gaussian behind the near plane: the reference traps in the
  kernel (antialias/cuda_rasterizer/auxiliary.h:157-160); here the forward returns
  FGS_ERR_PREFILTERED and the context stays usable.  The reference is not run on
  that input."""
import pytest
import torch

from _helpers import ours, small_case
from filtergs_b200 import _lib

pytestmark = pytest.mark.gpu


def _fwd(case, prefiltered=False):
    a = case.torch_inputs()
    a["prefiltered"] = prefiltered
    return ours.rasterize_gaussians(*a.values(), False, 0.2, 0.2, 0.05, 0.7, False)


def test_lookback_timeout_is_reported_and_context_survives(cuda):
    case = small_case(P=40000, seed=1201, W=320, H=240)
    clean = _fwd(case)
    torch.cuda.synchronize()
    try:
        # chunk 0 never publishes; its successors give up after 2 ms
        _lib.lib().fgs_debug_lookback_fault(0, 2_000_000)
        with pytest.raises(_lib.FgsError) as ei:
            _fwd(case)
        assert ei.value.status == _lib.FGS_ERR_TIMEOUT
    finally:
        _lib.lib().fgs_debug_lookback_fault(0xFFFFFFFF, 0)
    torch.cuda.synchronize()
    again = _fwd(case)
    torch.cuda.synchronize()
    assert again[0] == clean[0]
    for i in (1, 2, 3, 4, 5):
        assert torch.equal(again[i], clean[i]), i


def test_prefiltered_gaussian_behind_near_plane_is_an_error(cuda):
    case = small_case(P=3000, seed=1202, W=128, H=128)
    # every Gaussian in front of the near plane: prefiltered gives the same outputs
    base = _fwd(case)
    pre = _fwd(case, prefiltered=True)
    for i in (1, 2, 5):
        assert torch.equal(base[i], pre[i]), i
    # one Gaussian behind it (camera frame = world frame: z = 0.1 < 0.2)
    case.scene = dict(case.scene, means3D=case.scene["means3D"].copy())
    case.scene["means3D"][17] = (0.0, 0.0, 0.1)
    with pytest.raises(_lib.FgsError) as ei:
        _fwd(case, prefiltered=True)
    assert ei.value.status == _lib.FGS_ERR_PREFILTERED
    # the context is usable and the same input without prefiltered renders
    out = _fwd(case)
    torch.cuda.synchronize()
    assert out[0] > 0 and torch.isfinite(out[1]).all()
