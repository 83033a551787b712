"""CPU: the C oracle pinned against fixtures produced by the reference itself.

torchref_*.npz  -- the reference's own Python/torch code run on the CPU
                   (tests/golden/make_golden_torchref.py)
ref_*.npz       -- the reference's own CUDA build run on a B200
                   (tests/golden/make_golden_ref.py)

Integer outputs are compared exactly.  The forward preprocess of the oracle evaluates the
reference build's multiply-add grouping (fused where nvcc fused), so its per-Gaussian
floats match that build bit for bit; the rest of the oracle (radius, LoD, backward) keeps
plain float32 evaluation and is compared with a tolerance."""
import glob
import os

import numpy as np
import pytest

from _helpers import O, S

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def _load(name):
    p = os.path.join(GOLD, name)
    if not os.path.exists(p):
        pytest.fail(f"golden fixture {name} missing (regenerate with tests/golden/make_golden_*.py)")
    return np.load(p)


# ---------------------------------------------------------------- reference torch code
def test_radius_vs_reference_geometry():
    g = _load("torchref_geometry.npz")
    fx, fy = float(g["W"]) / (2 * float(g["tanfovx"])), float(g["H"]) / (2 * float(g["tanfovy"]))
    r = O.compute_radius(1, g["means3D"], g["scales"], g["rotations"], g["viewmatrix"].reshape(-1),
                         g["projmatrix"].reshape(-1), fx, fy, float(g["tanfovx"]), float(g["tanfovy"]))
    inside = r > 0                       # the torch version has no frustum cull
    assert inside.mean() > 0.9
    np.testing.assert_allclose(r[inside], g["radius"][inside], rtol=2e-6, atol=1e-6)


def test_activations_vs_reference():
    a = _load("torchref_activation.npz")
    N = a["xyz"].shape[0]
    idx = np.arange(N)
    for deg in (1, 2, 3):
        o = O.gather_activate(idx, a["xyz"], a["log_scale"], a["rot"], a["opacity"], a["dc"], a[f"rest{deg}"], deg,
                              a[f"campos{deg}"])
        np.testing.assert_allclose(o["scaling"], a[f"scaling{deg}"], rtol=1e-6)
        np.testing.assert_allclose(o["rotation"], a[f"rotation{deg}"], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(o["opacity"], a[f"opacity{deg}"], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(o["colors"], a[f"colors{deg}"], rtol=1e-5, atol=1e-6)


def test_ancestor_format_and_cut_order_vs_reference():
    t = _load("torchref_tree.npz")
    # the synthetic generator writes apps/ancestor.py's layout
    tr = S.lod_tree(P=20000, seed=2203, roots=3, max_depth=7, half_extent=60.0)
    assert np.array_equal(tr["ancestor_path"], t["ancestor_path"])
    assert np.array_equal(tr["node_index"], t["node_index"]) and np.array_equal(tr["tree"], t["tree"])
    # TensorTree.traverse order
    cut = O.log_cut(t["roots"], t["node_index"], t["tree"], t["radius"], 1.5)
    assert np.array_equal(cut, t["cut"])
    assert len(cut) > 1000


ANCESTOR_CASES = ["consistent", "noold", "messy", "oldkey", "chain", "err_parent", "err_width"]


@pytest.mark.parametrize("case", ANCESTOR_CASES)
def test_oracle_ancestor_path_vs_reference(case):
    """rebuild_ancestor_path (apps/ancestor.py) on consistent, inconsistent and failing trees."""
    a = _load("torchref_ancestor.npz")
    out = O.ancestor_path(a[case + "_parent"], a[case + "_depth"], int(a[case + "_width"]))
    if int(a[case + "_raises"]):
        assert out is None
    else:
        assert out is not None and np.array_equal(out, a[case + "_ancestor"])


# ---------------------------------------------------------------- reference CUDA build
def _raster_fixtures():
    return sorted(glob.glob(os.path.join(GOLD, "ref_*.npz")))


def _scene(d):
    colors = d["colors"] if d["colors"].shape[0] else None
    return O.Scene(d["means3D"], d["opacities"], int(d["W"]), int(d["H"]), float(d["tanfovx"]), float(d["tanfovy"]),
                   d["viewmatrix"].reshape(-1), d["projmatrix"].reshape(-1), d["campos"], bg=d["bg"],
                   shs=None if colors is not None else d["shs"], sh_degree=int(d["sh_degree"]) if colors is None else 0,
                   colors_precomp=colors, scales=d["scales"], rotations=d["rotations"],
                   use_filter=bool(d["use_filter"]))


@pytest.mark.parametrize("name", ["ref_sh3_filter.npz", "ref_colors_nofilter_ragged.npz", "ref_sh1_dense.npz"])
def test_oracle_forward_vs_reference_build(name):
    d = _load(name)
    sc = _scene(d)
    f = O.forward(sc)
    vis = d["radii"] > 0
    # The preprocess follows the reference build's multiply-add grouping, so every per-Gaussian
    # output is bit-identical; the binning and the per-pixel contributor counts follow from it.
    assert np.array_equal(f["pre"]["radii"], d["radii"])
    assert f["num_rendered"] == int(d["num_rendered"])
    for k in ("means2D", "depths", "conic_opacity"):
        assert np.array_equal(_bits(f["pre"][k][vis]), _bits(d["ref_" + k][vis])), k
    if d["colors"].size == 0:
        assert np.array_equal(_bits(f["pre"]["rgb"][vis]), _bits(d["ref_rgb"][vis]))
    assert np.array_equal(f["keys"].view(np.int64), d["ref_keys"]) or \
        np.array_equal(f["vals"].astype(np.int32), d["ref_vals"])
    assert np.array_equal(f["ranges"].astype(np.int32), d["ref_ranges"])
    assert np.array_equal(f["n_contrib"].astype(np.int32), d["ref_n_contrib"])
    # the host libm exp differs from the device exp in the last bit, which the blend carries
    np.testing.assert_allclose(f["color"], d["color"], rtol=0, atol=1e-6)


@pytest.mark.parametrize("name", ["ref_sh3_filter.npz", "ref_colors_nofilter_ragged.npz", "ref_sh1_dense.npz"])
def test_oracle_backward_vs_reference_build(name):
    d = _load(name)
    sc = _scene(d)
    f = O.forward(sc)
    b = O.backward(sc, f, d["dL"])
    for n in ("means2D", "colors", "opacity", "means3D", "cov3D", "sh", "scales", "rotations"):
        ref = d["grad_" + n]
        if ref.size == 0:
            continue
        mine = b[n].reshape(ref.shape)
        den = np.linalg.norm(ref)
        err = np.linalg.norm(mine - ref) / den if den > 0 else np.linalg.norm(mine)
        assert err <= 2e-4, (n, err)


def test_oracle_lod_mask_vs_reference_build():
    d = _load("ref_lod_tree.npz")
    mask, rad, dep = O.visibility_radius(d["xyz"], d["log_scales"], d["rotations"], d["projmatrix"].reshape(-1),
                                         d["viewmatrix"].reshape(-1), d["node_index"], d["ancestor_path"],
                                         float(d["fx"]), float(d["fy"]), float(d["tanfovx"]), float(d["tanfovy"]),
                                         float(d["padding"]), float(d["radius_max"]),
                                         float(d["radius_filter_threshold"]))
    assert np.mean(mask != d["mask"]) <= 1e-3
    assert mask.sum() > 0 and (~mask).sum() > 0
    np.testing.assert_allclose(rad, d["radius2d"], rtol=1e-5, atol=1e-5)
    # NDC depth = A - B / w cancels near the far plane; the GPU build contracts it into FMAs
    np.testing.assert_allclose(dep, d["depth"], rtol=1e-6, atol=1e-4)
    r = O.compute_radius(1, d["xyz"], d["scales_act"], d["rot_norm"], d["viewmatrix"].reshape(-1),
                         d["projmatrix"].reshape(-1), float(d["fx"]), float(d["fy"]), float(d["tanfovx"]),
                         float(d["tanfovy"]))
    np.testing.assert_allclose(r, d["radius_v2"], rtol=1e-5, atol=1e-5)


def test_fp32_vs_fp64_image_error_is_small():
    sc, cam = S.small_scene(P=3000, seed=2301, W=96, H=64)
    s = O.Scene(sc["means3D"], sc["opacities"], cam.W, cam.H, cam.tanfovx, cam.tanfovy, cam.viewmatrix.reshape(-1),
                cam.projmatrix.reshape(-1), cam.campos, shs=sc["shs"], sh_degree=3, scales=sc["scales"],
                rotations=sc["rotations"])
    f32, f64 = O.forward(s), O.forward(s, dtype=np.float64)
    assert np.abs(f32["color"] - f64["color"]).max() < 1e-3
