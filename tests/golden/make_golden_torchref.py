"""Generate golden fixtures from the reference's own Python/torch code (CPU).

Run where the reference tree is available (FGS_REFERENCE_ROOT, else a
`reference` directory beside this repository):

    python tests/golden/make_golden_torchref.py

Writes tests/golden/torchref_*.npz from:
  LoG/model/geometry.py      compute_radius (3-sigma radius with the 0.3 clamp)
  LoG/model/sh_utils.py      eval_sh_wobase + SH2RGB (colour activation)
  LoG/model/activation.py    exp / sigmoid / normalize activations
  apps/ancestor.py           rebuild_ancestor_path (the ancestor_path format)
  LoG/model/tensor_tree.py   TensorTree.traverse (the LoG cut order)
The CPU tests compare the C oracle (and the synthetic tree generator) with them.
"""
import importlib.util
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("FGS_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)

from filtergs_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _load(path, name):
    spec = importlib.util.spec_from_file_location(name, os.path.join(REF, path))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def geometry_case():
    from LoG.model import geometry
    sc, cam = S.small_scene(P=4000, seed=2201, W=160, H=120)
    camera = {"world_view_transform": torch.from_numpy(cam.viewmatrix), "FoVx": 2 * math.atan(cam.tanfovx),
              "FoVy": 2 * math.atan(cam.tanfovy), "image_height": cam.H, "image_width": cam.W}
    r = geometry.compute_radius(torch.from_numpy(sc["means3D"]), torch.from_numpy(sc["scales"]),
                                torch.from_numpy(sc["rotations"]), camera)
    np.savez_compressed(os.path.join(HERE, "torchref_geometry.npz"), means3D=sc["means3D"], scales=sc["scales"],
                        rotations=sc["rotations"], viewmatrix=cam.viewmatrix, projmatrix=cam.projmatrix,
                        W=cam.W, H=cam.H, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy, radius=r.numpy())


def activation_case():
    from LoG.model.activation import Activation
    rng = np.random.default_rng(2202)
    N = 600
    xyz = rng.uniform(-5, 5, (N, 3)).astype(np.float32)
    ls = rng.normal(-1, 1, (N, 3)).astype(np.float32)
    rot = rng.standard_normal((N, 4)).astype(np.float32)
    op = rng.normal(0, 2, (N, 1)).astype(np.float32)
    dc = rng.normal(0, 0.5, (N, 3)).astype(np.float32)
    out = {}
    for deg in (1, 2, 3):
        rest = rng.normal(0, 0.1, (N, (deg + 1) ** 2 - 1, 3)).astype(np.float32)
        campos = np.array([0.5, -1.0, 7.0], np.float32)
        ret = {"xyz": torch.from_numpy(xyz), "scaling": torch.from_numpy(ls), "rotation": torch.from_numpy(rot),
               "opacity": torch.from_numpy(op), "colors": torch.from_numpy(dc), "shs": torch.from_numpy(rest)}
        a = Activation().activate_root_return(ret, {"camera_center": torch.from_numpy(campos)}, deg)
        out[f"rest{deg}"] = rest
        out[f"campos{deg}"] = campos
        for k, v in a.items():
            out[f"{k}{deg}"] = v.numpy()
    np.savez_compressed(os.path.join(HERE, "torchref_activation.npz"), xyz=xyz, log_scale=ls, rot=rot, opacity=op,
                        dc=dc, **out)


def tree_case():
    anc_mod = _load("apps/ancestor.py", "ref_ancestor")
    from LoG.model.tensor_tree import TensorTree
    tr = S.lod_tree(P=20000, seed=2203, roots=3, max_depth=7, half_extent=60.0)
    sd = {"tree.index_parent": torch.from_numpy(tr["parent"]), "tree.depth": torch.from_numpy(tr["level"]).to(torch.int8)}
    anc, max_depth = anc_mod.rebuild_ancestor_path(sd)
    # LoG cut order with the v2 3-sigma radius of the activated parameters (the oracle computes it)
    c = tr["xyz"][tr["roots"]].mean(0)
    cam = S.look_at_camera(c + np.array([0.0, -140.0, 90.0]), c, W=320, H=180, fx=1600.0 / 6)
    fx, fy = cam.W / (2 * cam.tanfovx), cam.H / (2 * cam.tanfovy)
    scal = np.exp(tr["log_scales"])
    q = tr["rotations"] / np.maximum(np.linalg.norm(tr["rotations"], axis=1, keepdims=True), 1e-12)
    radius = O.compute_radius(1, tr["xyz"], scal, q, cam.viewmatrix.reshape(-1), cam.projmatrix.reshape(-1), fx, fy,
                              cam.tanfovx, cam.tanfovy)

    class Model:
        def compute_radius(self, index, camera, level=0):
            r = torch.from_numpy(radius)[index.long()]
            return r, r

    tree = TensorTree(max_child=tr["tree"].shape[1])
    tree.node_index = torch.from_numpy(tr["node_index"])
    tree.tree = torch.from_numpy(tr["tree"])
    tree.depth = torch.from_numpy(tr["level"]).to(torch.int8)
    tree.min_resolution_pixel = 1.5
    cut = tree.traverse(Model(), torch.from_numpy(tr["roots"]).long(), None)
    np.savez_compressed(os.path.join(HERE, "torchref_tree.npz"), parent=tr["parent"], level=tr["level"],
                        node_index=tr["node_index"], tree=tr["tree"], roots=tr["roots"], xyz=tr["xyz"],
                        log_scales=tr["log_scales"], rotations=tr["rotations"], viewmatrix=cam.viewmatrix,
                        projmatrix=cam.projmatrix, W=cam.W, H=cam.H, tanfovx=cam.tanfovx, tanfovy=cam.tanfovy,
                        ancestor_path=anc.numpy(), max_depth=max_depth, radius=radius, cut=cut.numpy())


def ancestor_case():
    """rebuild_ancestor_path on trees built to reach every branch of its level loop: a consistent
    tree with a wider stored table, the same without one (width = max depth + 1), a tree whose
    depths disagree with its parents' (orphans, parents in the same or a deeper level, depth-0
    nodes with parents, negative depths and parents), the old key name, and two inputs on which the
    reference raises (a parent id past the table, a depth past the stored width)."""
    anc_mod = _load("apps/ancestor.py", "ref_ancestor")
    rng = np.random.default_rng(2204)
    out = {}

    def run(name, parent, depth, old=None, key="tree.ancestor_path"):
        sd = {"tree.index_parent": torch.from_numpy(parent.astype(np.int32)),
              "tree.depth": torch.from_numpy(depth.astype(np.int8))}
        if old is not None:
            sd[key] = torch.from_numpy(old)
        out[name + "_parent"] = parent.astype(np.int32)
        out[name + "_depth"] = depth.astype(np.int32)
        out[name + "_width"] = np.int32(old.shape[1] if old is not None else (int(depth.max()) + 1 if depth.size else 1))
        try:
            anc, md = anc_mod.rebuild_ancestor_path(sd)
            out[name + "_ancestor"] = anc.numpy().astype(np.int32)
            out[name + "_max_depth"] = np.int32(md)
            out[name + "_raises"] = np.int32(0)
        except (IndexError, RuntimeError):
            out[name + "_raises"] = np.int32(1)

    tr = S.lod_tree(P=3000, seed=2205, roots=2, max_depth=5, half_extent=40.0)
    run("consistent", tr["parent"], tr["level"], old=np.zeros((3000, 8), np.int32))
    run("noold", tr["parent"], tr["level"])
    P = 2000
    parent = rng.integers(-3, P, P)
    depth = rng.integers(-1, 7, P)
    run("messy", parent, depth, old=np.zeros((P, 7), np.int32))
    run("oldkey", parent, depth, old=np.zeros((P, 9), np.int32), key="tree.ancestor")
    # a chain that climbs the levels in order, then nodes hanging off it at mixed depths
    chain = np.arange(-1, 9)
    run("chain", chain, np.arange(0, 10), old=np.zeros((10, 10), np.int32))
    bad = parent.copy()
    bad[17] = P + 5
    depth2 = depth.copy()
    depth2[17] = 3
    run("err_parent", bad, depth2, old=np.zeros((P, 7), np.int32))
    deep = depth.copy()
    deep[np.nonzero(parent >= 0)[0][0]] = 9
    run("err_width", parent, deep, old=np.zeros((P, 7), np.int32))
    np.savez_compressed(os.path.join(HERE, "torchref_ancestor.npz"), **out)


if __name__ == "__main__":
    geometry_case()
    activation_case()
    tree_case()
    ancestor_case()
    print("torchref fixtures written")
