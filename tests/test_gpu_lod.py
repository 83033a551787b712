"""GPU parity of the LoD selection path: the FilterGS visibility mask and radii
bit-exact against the reference build (oracle/_ref/ref_compute_radius_v2.so),
the gather bit-exact against ref_gather_attributes.so, the device LoG cut in
TensorTree.traverse order against the C oracle, culling and activation against
the oracle, and the selected-set render against the reference rasterizer."""
import numpy as np
import pytest
import torch

from _helpers import O, S, ref_gather_module, ref_module, ref_v2_module
from filtergs_b200 import filtergs_cuda as FC
from filtergs_b200 import lod

pytestmark = pytest.mark.gpu


def _tree(P=30000, seed=3101, roots=3, depth=8):
    tr = S.lod_tree(P=P, seed=seed, roots=roots, max_depth=depth, half_extent=60.0)
    c = tr["xyz"][tr["roots"]].mean(0)
    cam = S.look_at_camera(c + np.array([15.0, -150.0, 90.0]), c, W=640, H=360, fx=1600.0 / 3)
    return tr, cam


def _t(a, dt=None):
    x = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return x if dt is None else x.to(dt)


@pytest.fixture(scope="module")
def v2():
    m = ref_v2_module()
    if m is None:
        pytest.skip("reference build oracle/_ref/ref_compute_radius_v2.so not present")
    return m


def test_visibility_mask_bitexact_vs_reference(cuda, v2):
    for seed in (3101, 3102):
        tr, cam = _tree(seed=seed)
        fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
        args = (_t(tr["xyz"]), _t(tr["log_scales"]), _t(tr["rotations"]), _t(cam.projmatrix), _t(cam.viewmatrix),
                _t(tr["node_index"]), _t(tr["ancestor_path"]), fx, fy, cam.tanfovx, cam.tanfovy)
        for pad, rmax, thr in ((0.1, 1.5, 700.0), (0.5, 5.0, 0.0), (0.05, 2.0, 30.0)):
            a = FC.compute_radius_module.compute_visibility_radius(*args, pad, rmax, thr)
            b = v2.compute_visibility_radius(*args, pad, rmax, thr)
            assert torch.equal(a[0], b[0]), "mask"
            assert torch.equal(a[1], b[1]), "radius2d"
            assert torch.equal(a[2], b[2]), "depth"
            assert 0 < int(a[0].sum()) < tr["xyz"].shape[0]


def test_compute_radius_v2_bitexact_vs_reference(cuda, v2):
    tr, cam = _tree()
    fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
    sc = torch.exp(_t(tr["log_scales"]))
    rot = torch.nn.functional.normalize(_t(tr["rotations"]))
    args = (_t(tr["xyz"]), sc, rot, _t(cam.projmatrix), _t(cam.viewmatrix), fx, fy, cam.tanfovx, cam.tanfovy)
    assert torch.equal(FC.compute_radius_module.compute_radius(*args), v2.compute_radius(*args))


def test_gather_attributes_vs_reference(cuda):
    g = ref_gather_module()
    if g is None:
        pytest.skip("reference gather build not present")
    rng = np.random.default_rng(5)
    N, P = 5000, 20000
    idx = _t(rng.integers(0, P, N))
    xyz, sc, rot = _t(rng.standard_normal((P, 3), np.float32)), _t(rng.standard_normal((P, 3), np.float32)), \
        _t(rng.standard_normal((P, 4), np.float32))
    op, col, shs = _t(rng.standard_normal((P, 1), np.float32)), _t(rng.standard_normal((P, 3), np.float32)), \
        _t(rng.standard_normal((P, 15, 3), np.float32))
    a = FC.gather_attributes_cuda(idx, xyz, sc, rot, op, col, shs)
    b = g.gather_attributes_cuda(idx, xyz, sc, rot, op, col, shs)
    assert len(a) == len(b) == 6
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    d = FC.gather_attributes(idx, xyz, sc, rot, op, col)
    assert set(d) == {"xyz", "scaling", "rotation", "opacity", "colors"} and torch.equal(d["xyz"], b[0])


def test_compact_matches_nonzero(cuda):
    for n, p in ((1, 1.0), (255, 0.3), (256, 0.5), (100_003, 0.01), (1_000_000, 0.4)):
        m = torch.rand(n, device="cuda") < p
        idx, cnt = lod.compact(m)
        nz = torch.nonzero(m, as_tuple=True)[0]
        assert int(cnt.item()) == nz.numel()
        assert torch.equal(idx[:nz.numel()], nz)


def test_log_cut_order_matches_oracle(cuda):
    tr, cam = _tree(P=60000, seed=3103, roots=4, depth=9)
    scene = lod.TreeScene.from_arrays(tr)
    view, proj = _t(cam.viewmatrix), _t(cam.projmatrix)
    r = lod.node_radius(scene, view, proj, cam)
    ids, cnt = lod.log_cut(scene, r, 1.5, levels=30)
    n = int(cnt.item())
    o = O.log_cut(tr["roots"], tr["node_index"], tr["tree"], r.cpu().numpy(), 1.5)
    assert n == len(o) and n > 1000
    assert np.array_equal(ids[:n].cpu().numpy().astype(np.int64), o)
    # radius kernel on raw parameters vs the v2 kernel on torch-activated ones
    fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
    r2 = FC.compute_radius_module.compute_radius(scene.xyz, torch.exp(scene.log_scales),
                                                 torch.nn.functional.normalize(scene.rotations), proj, view, fx, fy,
                                                 cam.tanfovx, cam.tanfovy)
    # isotropic nodes make mid^2 - det a cancellation: an ulp in the quaternion norm moves the radius ~1e-5
    assert torch.allclose(r, r2, rtol=1e-4, atol=1e-4)
    # culling: order kept, radius < 1 px and opacity < 1/255 dropped
    out, oc = lod.cull(ids, cnt, r, scene.opacity_raw, 1.0)
    m = int(oc.item())
    sel = o[(r.cpu().numpy()[o] >= 1.0) & (1 / (1 + np.exp(-tr["opacity_raw"].reshape(-1)[o])) >= 1 / 255)]
    assert np.array_equal(out[:m].cpu().numpy(), sel)


def test_gather_activate_vs_oracle(cuda):
    tr, cam = _tree(P=20000, seed=3104)
    scene = lod.TreeScene.from_arrays(tr)
    idx = torch.randperm(scene.P, device="cuda")[:7000].sort().values
    cnt = torch.tensor([6000], dtype=torch.int64, device="cuda")
    rows = lod.gather_activate(scene, idx, cnt, _t(cam.campos), cap=7000)
    o = O.gather_activate(idx.cpu().numpy()[:6000], tr["xyz"], tr["log_scales"], tr["rotations"], tr["opacity_raw"],
                          tr["features_dc"], tr["shs_rest"], 1, cam.campos)
    for k, ok in (("xyz", "xyz"), ("scaling", "scaling"), ("rotation", "rotation"), ("opacity", "opacity"),
                  ("colors", "colors")):
        np.testing.assert_allclose(rows[k][:6000].cpu().numpy(), o[ok], rtol=2e-6, atol=2e-6)


@pytest.mark.parametrize("degenerate", [False, True])
def test_filtergs_selected_render_vs_reference_pipeline(cuda, v2, ref, degenerate):
    """The device path (mask -> compaction -> fused gather/activation -> row guard -> rasterizer)
    against the reference's own pieces (its visibility kernel, torch.nonzero, torch activations,
    FilterGS.render's finite/positive guard, its rasterizer).  `degenerate` gives some nodes an
    opacity whose sigmoid is 0 and a scale whose exp is 0, which the guard drops."""
    tr, cam = _tree(P=40000, seed=3105)
    if degenerate:
        tr = dict(tr, opacity_raw=tr["opacity_raw"].copy(), log_scales=tr["log_scales"].copy())
        tr["opacity_raw"].reshape(-1)[::37] = -1000.0
        tr["log_scales"][5::41, 1] = -300.0
    scene = lod.TreeScene.from_arrays(tr)
    view, proj, cpos = _t(cam.viewmatrix), _t(cam.projmatrix), _t(cam.campos)
    bg = torch.zeros(3, device="cuda")
    idx, cnt, mask, r2, dep = lod.select_filtergs(scene, view, proj, cam, 1.5, 0.1, 700.0)
    mine = lod.render_selected(scene, idx, cnt, view, proj, cpos, cam, bg)
    fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
    rm, _, _ = v2.compute_visibility_radius(scene.xyz, scene.log_scales, scene.rotations, proj, view,
                                            scene.node_index, scene.ancestor_path, fx, fy, cam.tanfovx, cam.tanfovy,
                                            0.1, 1.5, 700.0)
    ri = torch.nonzero(rm, as_tuple=True)[0]
    assert torch.equal(ri, idx[:int(cnt.item())])
    xyz = scene.xyz[ri]
    d = xyz - cpos[None]
    d = d / torch.norm(d, dim=-1, keepdim=True)
    rest = scene.shs_rest[ri]
    C0, C1 = 0.28209479177387814, 0.4886025119029199
    col = scene.features_dc[ri] * C0 + 0.5 + (-C1 * d[:, 1:2] * rest[:, 0] + C1 * d[:, 2:3] * rest[:, 1] -
                                              C1 * d[:, 0:1] * rest[:, 2])
    sc = torch.exp(scene.log_scales[ri])
    rot = torch.nn.functional.normalize(scene.rotations[ri])
    op = torch.sigmoid(scene.opacity_raw[ri])[:, None]
    # the fused gather + activation reproduces torch's op-by-op rounding (the norm's
    # summation order included), so the rasterizer sees the reference pipeline's bits
    rows = lod.gather_activate(scene, idx, cnt, cpos, cap=int(cnt.item()))
    assert torch.equal(rows["rotation"], rot)
    assert torch.equal(rows["scaling"], sc)
    assert torch.equal(rows["opacity"], op)
    assert torch.equal(rows["colors"], col)
    # FilterGS.render (FilterGS/filtergs.py:159-172)
    ok = (torch.isfinite(xyz).all(-1) & torch.isfinite(sc).all(-1) & torch.isfinite(rot).all(-1) &
          torch.isfinite(op).all(-1) & torch.isfinite(col).all(-1))
    ok = ok & (sc.min(dim=-1).values > 0.0) & (op[:, 0] > 0.0)
    assert bool(ok.all()) != degenerate
    xyz, col, op, sc, rot = xyz[ok], col[ok], op[ok], sc[ok], rot[ok]
    e = torch.Tensor([])
    theirs = ref.rasterize_gaussians(bg, xyz, col, op, sc, rot, 1.0, e, view, proj, cam.tanfovx, cam.tanfovy, cam.H,
                                     cam.W, e, 0, cpos, False, True, False, 0.2, 0.2, 0.05, 0.7, False)
    assert mine[0] == theirs[0], "num_rendered"
    assert torch.equal(mine[5], theirs[5]), "radii"
    assert torch.equal(mine[2], theirs[2]), "point_id"
    assert torch.equal(mine[1], theirs[1]), "image"


# ---------------------------------------------------------------- ancestor_path builder, checkpoints
ANCESTOR_CASES = ["consistent", "noold", "messy", "oldkey", "chain", "err_parent", "err_width"]


@pytest.mark.parametrize("case", ANCESTOR_CASES)
def test_ancestor_path_vs_reference(cuda, case):
    """fgs_ancestor_path against apps/ancestor.py's own output (tests/golden/torchref_ancestor.npz):
    consistent trees, trees whose depths disagree with their parents', and the two inputs on which
    the reference raises."""
    import os
    from filtergs_b200 import checkpoint as CK
    a = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "torchref_ancestor.npz"))
    par, dep, width = _t(a[case + "_parent"]), _t(a[case + "_depth"]), int(a[case + "_width"])
    if int(a[case + "_raises"]):
        with pytest.raises(IndexError):
            CK.ancestor_path_table(par, dep, width)
    else:
        out = CK.ancestor_path_table(par, dep, width)
        assert np.array_equal(out.cpu().numpy(), a[case + "_ancestor"])


def test_ancestor_path_large_tree_vs_generator(cuda):
    """2M-node tree: the device table equals the generator's (which the CPU tests pin to apps/ancestor.py)."""
    from filtergs_b200 import checkpoint as CK
    tr = S.lod_tree(P=2_000_000, seed=3111, roots=4, max_depth=11, half_extent=300.0)
    out = CK.ancestor_path_table(_t(tr["parent"]), _t(tr["level"]), tr["ancestor_path"].shape[1])
    assert torch.equal(out, _t(tr["ancestor_path"]))


def _log_state_dict(tr, with_ancestor):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    sd = {"gaussian.xyz": t(tr["xyz"]), "gaussian.scaling": t(tr["log_scales"]),
          "gaussian.rotation": t(tr["rotations"]), "gaussian.opacity": t(tr["opacity_raw"]),
          "gaussian.colors": t(tr["features_dc"]), "gaussian.shs": t(tr["shs_rest"]),
          "tree.root_index": t(tr["roots"]).to(torch.int32), "tree.node_index": t(tr["node_index"]),
          "tree.index_parent": t(tr["parent"]), "tree.depth": t(tr["level"]).to(torch.int8),
          "tree.tree": t(tr["tree"])}
    if with_ancestor:
        sd["tree.ancestor_path"] = t(tr["ancestor_path"])
    return sd


def test_checkpoint_without_ancestors_selects_like_the_arrays(cuda, tmp_path):
    """A LoG checkpoint with no ancestor table: the loader rebuilds it on the device and the
    FilterGS selection and render equal those of the scene built from the generator's arrays."""
    from filtergs_b200 import checkpoint as CK
    tr, cam = _tree(P=40000, seed=3112)
    path = tmp_path / "log.pth"
    torch.save({"state_dict": _log_state_dict(tr, with_ancestor=False), "global_iterations": 7}, path)
    sd = CK.load_statedict(str(path))
    scene = CK.tree_scene(sd, device="cuda")
    ref_scene = lod.TreeScene.from_arrays(tr, device="cuda")
    assert torch.equal(scene.ancestor_path, ref_scene.ancestor_path)
    view, proj, cpos = _t(cam.viewmatrix), _t(cam.projmatrix), _t(cam.campos)
    i1, c1, *_ = lod.select_filtergs(scene, view, proj, cam, 1.5, 0.1, 700.0)
    i2, c2, *_ = lod.select_filtergs(ref_scene, view, proj, cam, 1.5, 0.1, 700.0)
    n = int(c1.item())
    assert n == int(c2.item()) and n > 100 and torch.equal(i1[:n], i2[:n])
    bg = torch.zeros(3, device="cuda")
    r1 = lod.render_selected(scene, i1, c1, view, proj, cpos, cam, bg)
    r2 = lod.render_selected(ref_scene, i2, c2, view, proj, cpos, cam, bg)
    assert r1[0] == r2[0] and torch.equal(r1[1], r2[1])


def _eval_sh_wobase_torch(dirs, sh, degree):
    """LoG/model/sh_utils.py:31-68 as the reference runs it: torch element-wise ops, in its order."""
    C1 = 0.4886025119029199
    C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
    C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
          1.445305721320277, -0.5900435899266435]
    x, y, z = dirs[..., 0:1], dirs[..., 1:2], dirs[..., 2:3]
    result = - C1 * y * sh[..., 0, :] + C1 * z * sh[..., 1, :] - C1 * x * sh[..., 2, :]
    if degree > 1:
        xx, yy, zz = x * x, y * y, z * z
        xy, yz, xz = x * y, y * z, x * z
        result = (result + C2[0] * xy * sh[..., 3, :] + C2[1] * yz * sh[..., 4, :] +
                  C2[2] * (2.0 * zz - xx - yy) * sh[..., 5, :] + C2[3] * xz * sh[..., 6, :] +
                  C2[4] * (xx - yy) * sh[..., 7, :])
        if degree > 2:
            result = (result + C3[0] * y * (3 * xx - yy) * sh[..., 8, :] + C3[1] * xy * z * sh[..., 9, :] +
                      C3[2] * y * (4 * zz - xx - yy) * sh[..., 10, :] +
                      C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * sh[..., 11, :] +
                      C3[4] * x * (4 * zz - xx - yy) * sh[..., 12, :] + C3[5] * z * (xx - yy) * sh[..., 13, :] +
                      C3[6] * x * (xx - 3 * yy) * sh[..., 14, :])
    return result


@pytest.mark.parametrize("deg", [1, 2, 3])
def test_gather_activate_bitexact_vs_torch_activation(cuda, deg):
    """The fused gather + activation against LoG/model/activation.py:36-43 run as torch ops on the
    gathered rows (exp, sigmoid, F.normalize, SH2RGB + eval_sh_wobase): equal bit for bit."""
    tr, cam = _tree(P=30000, seed=3120 + deg)
    rest = np.random.default_rng(deg).normal(0, 0.2, (tr["xyz"].shape[0], (deg + 1) ** 2 - 1, 3)).astype(np.float32)
    scene = lod.TreeScene(tr["xyz"], tr["log_scales"], tr["rotations"], tr["opacity_raw"], tr["features_dc"], rest,
                          tr["node_index"], tr["ancestor_path"], tr["tree"], tr["roots"], sh_degree=deg)
    cpos = _t(cam.campos)
    idx = torch.randperm(scene.P, device="cuda")[:12000].sort().values
    cnt = torch.tensor([12000], dtype=torch.int64, device="cuda")
    rows = lod.gather_activate(scene, idx, cnt, cpos, cap=12000)
    xyz = scene.xyz[idx]
    d = xyz - cpos[None]
    d = d / torch.norm(d, dim=-1, keepdim=True)
    colors = scene.features_dc[idx] * 0.28209479177387814 + 0.5
    colors = colors + _eval_sh_wobase_torch(d, scene.shs_rest[idx], deg)
    assert torch.equal(rows["xyz"], xyz)
    assert torch.equal(rows["scaling"], torch.exp(scene.log_scales[idx]))
    assert torch.equal(rows["rotation"], torch.nn.functional.normalize(scene.rotations[idx]))
    assert torch.equal(rows["opacity"].reshape(-1), torch.sigmoid(scene.opacity_raw[idx]))
    assert torch.equal(rows["colors"], colors)
