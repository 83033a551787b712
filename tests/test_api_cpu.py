"""CPU: the Python operator API mirrors the reference's surface
(antialias/diff_gaussian_rasterization_wodilate/__init__.py)."""
import sys

import pytest
import torch

import filtergs_b200
from filtergs_b200 import rasterization as R
from filtergs_b200.diff_gaussian_rasterization_wodilate import (GaussianRasterizationSettings, GaussianRasterizer,
                                                                _RasterizeGaussians, rasterize_gaussians)


def _settings(**kw):
    z = torch.zeros(3)
    return GaussianRasterizationSettings(32, 48, 0.5, 0.4, z, 1.0, torch.eye(4), torch.eye(4), 0, z, False, False, **kw)


def test_settings_fields_and_defaults():
    s = _settings()
    ref_fields = ("image_height", "image_width", "tanfovx", "tanfovy", "bg", "scale_modifier", "viewmatrix",
                  "projmatrix", "sh_degree", "campos", "prefiltered", "debug", "ogfs_epsilon_scale",
                  "ogfs_epsilon_max", "ogfs_energy_floor", "ogfs_radius_ratio_min", "ogfs_enable_stats")
    assert GaussianRasterizationSettings._fields[:len(ref_fields)] == ref_fields
    assert (s.ogfs_epsilon_scale, s.ogfs_epsilon_max, s.ogfs_energy_floor, s.ogfs_radius_ratio_min,
            s.ogfs_enable_stats) == (0.2, 0.2, 0.05, 0.7, True)
    assert s.filter3d_scale == 0.0 and s.backward_mode == "ref_compat"
    assert s._replace(ogfs_epsilon_scale=0.5).ogfs_epsilon_scale == 0.5   # apps/render.py overrides this way


def test_rasterizer_argument_checks_match_reference():
    r = GaussianRasterizer(_settings())
    m = torch.zeros(4, 3)
    with pytest.raises(Exception, match="excatly one of either SHs or precomputed colors"):
        r(m, m, torch.ones(4, 1), scales=m, rotations=torch.zeros(4, 4))
    with pytest.raises(Exception, match="exactly one of either scale/rotation pair or precomputed 3D covariance"):
        r(m, m, torch.ones(4, 1), colors_precomp=m)
    with pytest.raises(Exception, match="exactly one of either scale/rotation"):
        r(m, m, torch.ones(4, 1), colors_precomp=m, scales=m, rotations=torch.zeros(4, 4),
          cov3D_precomp=torch.zeros(4, 6))


def test_rasterize_needs_cuda_tensors():
    from filtergs_b200 import _C
    z = torch.zeros(3)
    with pytest.raises(RuntimeError, match="CUDA"):
        _C.rasterize_gaussians(z, torch.zeros(5, 3), torch.Tensor([]), torch.ones(5, 1), torch.ones(5, 3),
                               torch.zeros(5, 4), 1.0, torch.Tensor([]), torch.eye(4), torch.eye(4), 0.5, 0.5, 16, 16,
                               torch.zeros(5, 1, 3), 0, z, False, True)
    with pytest.raises(RuntimeError, match="num_points, 3"):
        _C.rasterize_gaussians(z, torch.zeros(5, 2), torch.Tensor([]), torch.ones(5, 1), torch.ones(5, 3),
                               torch.zeros(5, 4), 1.0, torch.Tensor([]), torch.eye(4), torch.eye(4), 0.5, 0.5, 16, 16,
                               torch.zeros(5, 1, 3), 0, z, False, True)


def test_latest_stats_parsing_matches_reference_layout():
    T = 6
    v = torch.zeros(9 + 128 + 2 * T, dtype=torch.float64)
    v[0], v[3], v[4], v[5], v[6], v[7], v[8] = 0.25, 100, T, 40, 70, 30, 11
    v[9:20] = torch.arange(11) + 1
    v[9 + 64:9 + 64 + 11] = 5
    v[9 + 128:9 + 128 + T] = 0.5
    v[9 + 128 + T:] = 7
    d = R.parse_stats(v)
    assert d["bar_g"] == 0.25 and d["num_tiles"] == T and d["num_kpc_bins"] == 11
    assert d["kpc_edges"] == [float(i + 1) for i in range(11)] and d["kpc_hist"] == [5.0] * 11
    assert d["tile_ratio"] == [0.5] * T and d["tile_total_kv"] == [7.0] * T
    assert R.parse_stats(torch.zeros(5, dtype=torch.float64)) is None


def test_autograd_function_arity():
    # forward takes the reference's 15 inputs; backward returns one gradient slot per input
    import inspect
    assert len(inspect.signature(_RasterizeGaussians.forward).parameters) == 16  # ctx + 15
    assert len(inspect.signature(rasterize_gaussians).parameters) == 15


def test_install_dropin():
    dgr = filtergs_b200.install_dropin()
    assert sys.modules["diff_gaussian_rasterization_wodilate"] is dgr
    import diff_gaussian_rasterization_wodilate as alias
    assert alias.GaussianRasterizer is GaussianRasterizer


def test_checkpoint_loader_on_cpu(tmp_path):
    """LoG checkpoint parsing (LoG/utils/command.py:12-16 unwrap, the gaussian.* / tree.* keys) with a
    stored ancestor table; the rebuild itself is a device pass and refuses a CPU device."""
    import numpy as np
    from filtergs_b200 import checkpoint as CK
    from filtergs_b200 import synthetic as S
    tr = S.lod_tree(P=500, seed=41, roots=2, max_depth=4, half_extent=20.0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    sd = {"gaussian.xyz": t(tr["xyz"]), "gaussian.scaling": t(tr["log_scales"]),
          "gaussian.rotation": t(tr["rotations"]), "gaussian.opacity": t(tr["opacity_raw"]),
          "gaussian.colors": t(tr["features_dc"]), "gaussian.shs": t(tr["shs_rest"]),
          "tree.root_index": t(tr["roots"]).to(torch.int32), "tree.node_index": t(tr["node_index"]),
          "tree.index_parent": t(tr["parent"]), "tree.depth": t(tr["level"]).to(torch.int8),
          "tree.tree": t(tr["tree"]), "tree.ancestor": t(tr["ancestor_path"])}
    for wrapped in (True, False):
        path = tmp_path / f"c{int(wrapped)}.pth"
        torch.save({"state_dict": sd, "global_iterations": 3} if wrapped else sd, path)
        got = CK.load_statedict(str(path))
        assert set(got) == set(sd)
        scene = CK.tree_scene(got, device="cpu")
        assert scene.P == 500 and scene.sh_degree == 1
        assert torch.equal(scene.ancestor_path, t(tr["ancestor_path"]))
        assert torch.equal(scene.opacity_raw, t(tr["opacity_raw"]).reshape(-1))
    assert CK.tree_scene(sd, device="cpu", sh_degree=0).shs_rest is None
    with pytest.raises(ValueError):
        CK.tree_scene(sd, device="cpu", sh_degree=2)
    with pytest.raises(ValueError):
        CK.tree_scene(sd, device="cpu", rebuild_ancestors=True)   # the builder runs on a GPU only
    bare = {k: v for k, v in sd.items() if k != "tree.ancestor"}
    with pytest.raises(KeyError):
        CK.tree_scene(bare, device="cpu", rebuild_ancestors=False)
    with pytest.raises(KeyError):
        CK.rebuild_ancestor_path({"tree.depth": sd["tree.depth"]})
    assert CK.sh_degree_of(torch.zeros(4, 15, 3)) == 3 and CK.sh_degree_of(None) == 0
    with pytest.raises(ValueError):
        CK.sh_degree_of(torch.zeros(4, 5, 3))
