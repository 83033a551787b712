"""FP64 central-difference gradients of L = sum(dL * image) through the C oracle.

The renderer is piecewise smooth: tile culling, the alpha >= 1/255 and
T >= 1e-4 cut-offs and the 0.99 / 0.3 clamps are discontinuities.  Each
parameter is differenced with h and h/2; a parameter whose two estimates
disagree straddles a discontinuity and is reported as such instead of being
compared."""
import numpy as np

from _helpers import O

FIELDS = ("means3D", "scales", "rotations", "opacities", "shs")


def pick_params(scene, radii, n, seed):
    rng = np.random.default_rng(seed)
    vis = np.nonzero(radii > 0)[0]
    out = []
    for _ in range(n):
        f = FIELDS[rng.integers(len(FIELDS))]
        i = int(rng.choice(vis))
        shape = scene[f].shape[1:]
        comp = tuple(int(rng.integers(s)) for s in shape)
        out.append((f, i, comp))
    return out


def make_scene(scene, cam, bg=(0.0, 0.0, 0.0), use_filter=True):
    return O.Scene(scene["means3D"], scene["opacities"], cam.W, cam.H, cam.tanfovx, cam.tanfovy,
                   cam.viewmatrix.reshape(-1), cam.projmatrix.reshape(-1), cam.campos, bg=bg, shs=scene["shs"],
                   sh_degree=scene["sh_degree"], scales=scene["scales"], rotations=scene["rotations"],
                   use_filter=use_filter)


def loss64(scene, cam, dL, bg, use_filter):
    s64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in scene.items()}
    f = O.forward(make_scene(s64, cam, bg, use_filter), dtype=np.float64)
    return float((f["color"] * dL).sum())


def fd(scene, cam, dL, params, rel_h=1e-4, bg=(0.0, 0.0, 0.0), use_filter=True):
    """[(fd, consistent)] per parameter."""
    res = []
    base = {k: (np.array(v, np.float64) if isinstance(v, np.ndarray) else v) for k, v in scene.items()}
    dL = dL.astype(np.float64)
    for f, i, comp in params:
        theta = base[f][(i,) + comp]
        est = []
        for h in (rel_h * max(1.0, abs(theta)), 0.5 * rel_h * max(1.0, abs(theta))):
            vals = []
            for sgn in (1.0, -1.0):
                s = dict(base)
                s[f] = base[f].copy()
                s[f][(i,) + comp] = theta + sgn * h
                vals.append(loss64(s, cam, dL, bg, use_filter))
            est.append((vals[0] - vals[1]) / (2 * h))
        a, b = est
        ok = abs(a - b) <= 1e-3 * max(abs(a), abs(b)) + 1e-6
        res.append((b, ok))
    return res
