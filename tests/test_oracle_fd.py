"""CPU: the oracle's FP64 backward in `consistent` mode equals FP64 central
differences of its own forward (the derivation the CUDA backward follows)."""
import numpy as np

from _fd import fd, make_scene, pick_params
from _helpers import O, S


def test_consistent_backward_matches_central_differences_fp64():
    sc, cam = S.small_scene(P=1500, seed=4001, W=64, H=48)
    rng = np.random.default_rng(4002)
    dL = rng.standard_normal((3, cam.H, cam.W))
    s64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in sc.items()}
    osc = make_scene(s64, cam)
    f = O.forward(osc, dtype=np.float64)
    g = O.backward(osc, f, dL, dtype=np.float64, consistent=True)
    params = pick_params(sc, f["pre"]["radii"], 24, seed=4003)
    res = fd(sc, cam, dL, params)
    names = {"means3D": "means3D", "scales": "scales", "rotations": "rotations", "opacities": "opacity",
             "shs": "sh"}
    checked = 0
    scale = np.sqrt(np.mean([r[0] ** 2 for r in res])) + 1e-12
    for (fname, i, comp), (num, smooth) in zip(params, res):
        if not smooth:
            continue
        ana = g[names[fname]].reshape((g[names[fname]].shape[0],) + sc[fname].shape[1:])[(i,) + comp]
        assert abs(ana - num) <= 1e-5 * max(abs(num), 1e-3 * scale), (fname, i, comp, ana, num)
        checked += 1
    assert checked >= 20
